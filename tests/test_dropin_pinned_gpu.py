"""GPU: how the drop-in calls move the FP64 embeddings.

By default (with at least 4 host threads) the host threads convert only the
rows of the words that occur in the target matrix or in r to FP32 into
pinned memory and copy those (4 bytes per entry instead of 8).  With
WMD_DROPIN_NARROW=0, pinned embeddings are read in place by the GPU (the
same rows, in FP64) and pageable ones are copied whole.  The results must be
bit-identical on every path (the FP64 -> FP32 rounding is the same and the
solve never touches any other row), and ``wmd_dropin_h2d_bytes`` must count
exactly the bytes that crossed the bus.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

# the library narrows on the host when OpenMP has at least 4 threads
NARROW = int(os.environ.get("OMP_NUM_THREADS") or len(os.sched_getaffinity(0))) >= 4


def _bytes(V, d, N, nnz, rows):
    # target matrix (col_ptr, rows, vals) + length order + r + embedding rows
    return (N + 1) * 8 + nnz * 16 + N * 4 + V * 8 + rows * d * 8


def _bytes_narrow(V, d, N, nnz, rows):
    # the same with the slot map (int32 per word) and FP32 rows
    return (N + 1) * 8 + nnz * 16 + N * 4 + V * 8 + V * 4 + rows * d * 4


@pytest.mark.parametrize("params", [
    (3000, 300, 60, 32, 8, 128, 50, 70),           # v_r = 32
    (2000, 7, 80, 20, 4, 40, 30, 71, 10.0, 15, 5),  # d = 7, empty documents
])
def test_pinned_embeddings_read_only_needed_rows(wmd, synth, params, monkeypatch):
    p = synth.case(*params)
    V, d = p.vecs.shape
    N = p.col_ptr.size - 1
    vecs = np.ascontiguousarray(p.vecs, np.float64)
    args = (p.col_ptr, p.row_inds, p.vals)
    used = np.union1d(np.unique(p.row_inds), np.flatnonzero(p.r))
    assert used.size < V
    pin = torch.from_numpy(vecs.copy()).pin_memory()
    for variant, lam in (("fused", -p.lam), ("nonfused", p.lam)):
        # default: rows narrowed on the host, pageable or pinned alike
        narrowed = wmd.sinkhorn_wmd_csc(p.r, vecs, *args, lam, p.max_iter, variant)
        nb = wmd.dropin_h2d_bytes()
        narrowed_pin = wmd.sinkhorn_wmd_csc(p.r, pin.numpy(), *args, lam, p.max_iter,
                                            variant)
        np.testing.assert_array_equal(narrowed_pin, narrowed)
        if NARROW:
            assert nb == _bytes_narrow(V, d, N, p.row_inds.size, used.size)
            assert wmd.dropin_h2d_bytes() == nb
        # device-side paths
        monkeypatch.setenv("WMD_DROPIN_NARROW", "0")
        pageable = wmd.sinkhorn_wmd_csc(p.r, vecs, *args, lam, p.max_iter, variant)
        full = wmd.dropin_h2d_bytes()
        pinned = wmd.sinkhorn_wmd_csc(p.r, pin.numpy(), *args, lam, p.max_iter, variant)
        part = wmd.dropin_h2d_bytes()
        monkeypatch.delenv("WMD_DROPIN_NARROW")
        np.testing.assert_array_equal(pinned, pageable)
        np.testing.assert_array_equal(narrowed, pageable)
        assert full == _bytes(V, d, N, p.row_inds.size, V)
        assert part == _bytes(V, d, N, p.row_inds.size, used.size)


def test_pinned_view_at_an_offset_and_csr_drop_in(wmd, synth, monkeypatch):
    """A view into a larger pinned buffer is read in place as well; the CSR
    drop-in (the reference's own call shape) takes the same path."""
    monkeypatch.setenv("WMD_DROPIN_NARROW", "0")
    p = synth.case(3000, 300, 60, 32, 8, 128, 50, 70)
    V, d = p.vecs.shape
    N = p.col_ptr.size - 1
    vecs = np.ascontiguousarray(p.vecs, np.float64)
    big = torch.zeros(V + 7, d, dtype=torch.float64).pin_memory()
    big[5:5 + V] = torch.from_numpy(vecs)
    view = big[5:5 + V].numpy()
    ref = wmd.sinkhorn_wmd_csc(p.r, vecs, p.col_ptr, p.row_inds, p.vals,
                               -p.lam, p.max_iter)
    got = wmd.sinkhorn_wmd_csc(p.r, view, p.col_ptr, p.row_inds, p.vals,
                               -p.lam, p.max_iter)
    np.testing.assert_array_equal(got, ref)
    used = np.union1d(np.unique(p.row_inds), np.flatnonzero(p.r))
    assert wmd.dropin_h2d_bytes() == _bytes(V, d, N, p.row_inds.size, used.size)
    # word-major CSR, as the reference's sinkhorn_wmd takes it
    rows = np.repeat(np.arange(N), np.diff(p.col_ptr))
    order = np.lexsort((rows, p.row_inds))
    row_ptr = np.zeros(V + 1, np.int64)
    np.add.at(row_ptr, p.row_inds + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    csr_args = (-p.lam, p.max_iter, row_ptr, rows[order], p.vals[order], N)
    csr_pageable = wmd.sinkhorn_wmd_fused(p.r, vecs, *csr_args)
    csr_pinned = wmd.sinkhorn_wmd_fused(p.r, view, *csr_args)
    np.testing.assert_array_equal(csr_pinned, csr_pageable)
    np.testing.assert_allclose(csr_pinned, ref, rtol=1e-5)
    # rows narrowed on the host: the same scores
    monkeypatch.delenv("WMD_DROPIN_NARROW")
    np.testing.assert_array_equal(wmd.sinkhorn_wmd_fused(p.r, view, *csr_args), csr_pinned)
