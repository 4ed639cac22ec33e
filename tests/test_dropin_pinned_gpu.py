"""GPU: drop-in calls whose FP64 embeddings sit in pinned host memory.

The GPU then reads only the rows of the words that occur in the target matrix
or in r, directly from host memory, instead of copying the whole V x d matrix.
The results must be bit-identical to the copying path (the solve never touches
any other row), and ``wmd_dropin_h2d_bytes`` must count exactly the bytes that
crossed the bus.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bytes(V, d, N, nnz, rows):
    # target matrix (col_ptr, rows, vals) + length order + r + embedding rows
    return (N + 1) * 8 + nnz * 16 + N * 4 + V * 8 + rows * d * 8


@pytest.mark.parametrize("params", [
    (3000, 300, 60, 32, 8, 128, 50, 70),           # v_r = 32
    (2000, 7, 80, 20, 4, 40, 30, 71, 10.0, 15, 5),  # d = 7, empty documents
])
def test_pinned_embeddings_read_only_needed_rows(wmd, synth, params):
    p = synth.case(*params)
    V, d = p.vecs.shape
    N = p.col_ptr.size - 1
    vecs = np.ascontiguousarray(p.vecs, np.float64)
    args = (p.col_ptr, p.row_inds, p.vals)
    for variant, lam in (("fused", -p.lam), ("nonfused", p.lam)):
        pageable = wmd.sinkhorn_wmd_csc(p.r, vecs, *args, lam, p.max_iter, variant)
        full = wmd.dropin_h2d_bytes()
        pin = torch.from_numpy(vecs.copy()).pin_memory()
        pinned = wmd.sinkhorn_wmd_csc(p.r, pin.numpy(), *args, lam, p.max_iter, variant)
        part = wmd.dropin_h2d_bytes()
        np.testing.assert_array_equal(pinned, pageable)
        used = np.union1d(np.unique(p.row_inds), np.flatnonzero(p.r))
        assert full == _bytes(V, d, N, p.row_inds.size, V)
        assert part == _bytes(V, d, N, p.row_inds.size, used.size)
        assert used.size < V


def test_pinned_view_at_an_offset_and_csr_drop_in(wmd, synth):
    """A view into a larger pinned buffer is read in place as well; the CSR
    drop-in (the reference's own call shape) takes the same path."""
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
