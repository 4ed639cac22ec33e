"""GPU: the allocation-free entry point wmd_sinkhorn_noalloc.

It exists for callers that may not allocate device memory (a framework or
inference server that owns all device memory and hands plugins only their
input and output buffers, or a latency-critical loop that cannot take the
device-wide synchronisation of cudaMalloc / cudaFree).  Its working buffers
live in a fixed scratch array inside the library, shared by every call.

The tests call it through the C ABI with caller-owned device buffers, twice
in a row (the second call reuses the scratch the first one left behind), and
check both results against the FP64 oracle within the plain path's
tolerance; they check that calls after the first one leave the device's free
memory unchanged, and that refused arguments come back as a status.  The
file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same bar as the plain path's parity tests
WMD_ERR_INVALID_ARG = 1


def _call(wmd, p, bufs, stream=None, E=None, vr_cap=None):
    r, E0, cp, ri, vv, out = bufs
    E = E0.data_ptr() if E is None else E
    return wmd.lib().wmd_sinkhorn_noalloc(
        ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(E), p.V, p.d,
        ctypes.c_void_p(cp.data_ptr()), ctypes.c_void_p(ri.data_ptr()),
        ctypes.c_void_p(vv.data_ptr()), p.N, p.nnz,
        p.v_r if vr_cap is None else vr_cap, p.lam, p.max_iter,
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))


def _bufs(p):
    import torch
    dev = torch.device("cuda", 0)
    r = torch.from_numpy(p.r).to(dev)
    E = torch.from_numpy(p.vecs).to(dev)
    cp = torch.from_numpy(p.col_ptr.astype(np.int64)).to(dev)
    ri = torch.from_numpy(p.row_inds.astype(np.int64)).to(dev)
    vv = torch.from_numpy(p.vals).to(dev)
    out = torch.full((p.N,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    return r, E, cp, ri, vv, out


def _oracle(oracle_mod, p):
    return oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                               p.row_inds, p.vals, p.lam, p.max_iter)


@pytest.mark.parametrize("case", ["small", "single_source"])
def test_noalloc_matches_oracle_twice(wmd, synth, oracle_mod, case):
    if case == "small":
        p = synth.case(3000, 300, 300, 32, 8, 200, 50, 77)
    else:
        p = synth.single_source()  # V=1e5, d=300, v_r=32, N=5000
    ref = _oracle(oracle_mod, p)
    bufs = _bufs(p)
    for call in range(2):
        bufs[-1].fill_(float("nan"))
        st = _call(wmd, p, bufs)
        assert st == 0, wmd.lib().wmd_last_error()
        got = bufs[-1].cpu().numpy()
        err = rel_err(got, ref)
        assert err.max() <= TOL, f"call {call}: max rel err {err.max():.3e}"


def test_noalloc_allocates_nothing(wmd, synth, oracle_mod):
    """After the first call on the device (which loads the kernels and looks
    up the scratch address), further calls leave the free device memory
    exactly where it was."""
    import torch
    p = synth.case(4000, 300, 200, 24, 8, 160, 50, 79)
    ref = _oracle(oracle_mod, p)
    bufs = _bufs(p)
    assert _call(wmd, p, bufs) == 0, wmd.lib().wmd_last_error()
    torch.cuda.synchronize()
    for call in range(3):
        free0, _ = torch.cuda.mem_get_info(0)
        st = _call(wmd, p, bufs)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(0)
        assert st == 0, wmd.lib().wmd_last_error()
        assert free1 == free0, f"call {call}: free memory moved by {free0 - free1} bytes"
    err = rel_err(bufs[-1].cpu().numpy(), ref)
    assert err.max() <= TOL


def test_noalloc_rejects_problems_beyond_its_scratch(wmd, synth):
    p = synth.case(3000, 300, 50, 32, 8, 64, 50, 78)
    bufs = _bufs(p)
    r, E, cp, ri, vv, out = bufs
    # Pretend the vocabulary is huge: the size check fires before any
    # device work, so the undersized buffers are never touched.
    st = wmd.lib().wmd_sinkhorn_noalloc(
        ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(E.data_ptr()),
        2_000_000, p.d, ctypes.c_void_p(cp.data_ptr()),
        ctypes.c_void_p(ri.data_ptr()), ctypes.c_void_p(vv.data_ptr()), p.N,
        p.nnz, 512, p.lam, p.max_iter, ctypes.c_void_p(out.data_ptr()), None)
    assert st == WMD_ERR_INVALID_ARG
    assert b"scratch" in wmd.lib().wmd_last_error()
    # absurd sizes whose byte counts would wrap around are refused too
    st = wmd.lib().wmd_sinkhorn_noalloc(
        ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(E.data_ptr()),
        p.V, p.d, ctypes.c_void_p(cp.data_ptr()),
        ctypes.c_void_p(ri.data_ptr()), ctypes.c_void_p(vv.data_ptr()), p.N,
        1 << 62, 32, p.lam, p.max_iter, ctypes.c_void_p(out.data_ptr()), None)
    assert st == WMD_ERR_INVALID_ARG
    # and the entry point still works afterwards
    assert _call(wmd, p, bufs) == 0


def test_noalloc_refuses_misaligned_embeddings(wmd, synth, oracle_mod):
    """d % 4 == 0 takes 16-byte vector loads of the embeddings: a base that
    is only 4-byte aligned (a slice of a larger buffer) is refused with a
    status before any kernel runs."""
    import torch
    p = synth.case(3000, 300, 50, 32, 8, 64, 50, 80)
    bufs = _bufs(p)
    E = bufs[1]
    shifted = torch.empty(E.numel() + 4, dtype=torch.float32, device=E.device)
    shifted[1:1 + E.numel()] = E.reshape(-1)
    torch.cuda.synchronize()
    st = _call(wmd, p, bufs, E=shifted.data_ptr() + 4)
    assert st == WMD_ERR_INVALID_ARG
    assert b"aligned" in wmd.lib().wmd_last_error()
    assert _call(wmd, p, bufs) == 0
    err = rel_err(bufs[-1].cpu().numpy(), _oracle(oracle_mod, p))
    assert err.max() <= TOL
