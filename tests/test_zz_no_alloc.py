"""GPU: the allocation-free entry point wmd_sinkhorn_noalloc.

It exists for callers that may not allocate device memory (a framework or
inference server that owns all device memory and hands plugins only their
input and output buffers, or a latency-critical loop that cannot take the
device-wide synchronisation of cudaMalloc / cudaFree).  Its working buffers
live in a fixed scratch array inside the library, shared by every call.

This test calls it through the C ABI with caller-owned device buffers, twice
in a row (the second call reuses the scratch the first one left behind), and
checks both results against the regular drop-in entry point within the plain
path's tolerance.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same bar as the plain path's parity tests


def _call(wmd, p, bufs, stream=None):
    import torch
    r, E, cp, ri, vv, out = bufs
    st = wmd.lib().wmd_sinkhorn_noalloc(
        ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(E.data_ptr()), p.V, p.d,
        ctypes.c_void_p(cp.data_ptr()), ctypes.c_void_p(ri.data_ptr()),
        ctypes.c_void_p(vv.data_ptr()), p.N, p.nnz, p.v_r, p.lam, p.max_iter,
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    return st


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


@pytest.mark.parametrize("case", ["small", "single_source"])
def test_noalloc_matches_regular_entry_twice(wmd, synth, case):
    if case == "small":
        p = synth.case(3000, 300, 300, 32, 8, 200, 50, 77)
    else:
        p = synth.single_source()  # V=1e5, d=300, v_r=32, N=5000
    ref = wmd.sinkhorn_wmd_csc(p.r, p.vecs.astype(np.float64), p.col_ptr,
                               p.row_inds, p.vals, -p.lam, p.max_iter, "fused")
    bufs = _bufs(p)
    for call in range(2):
        bufs[-1].fill_(float("nan"))
        st = _call(wmd, p, bufs)
        assert st == 0, wmd.lib().wmd_last_error()
        got = bufs[-1].cpu().numpy()
        err = rel_err(got, ref)
        assert err.max() <= TOL, f"call {call}: max rel err {err.max():.3e}"


def test_noalloc_rejects_problems_beyond_its_scratch(wmd, synth):
    import torch
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
    assert st == 1  # WMD_ERR_INVALID_ARG
    assert b"scratch" in wmd.lib().wmd_last_error()
    # and the entry point still works afterwards
    assert _call(wmd, p, bufs) == 0
