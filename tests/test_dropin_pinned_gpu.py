"""GPU: how the drop-in calls move the FP64 embeddings.

With the embeddings in pinned (device-mapped) host memory, the host threads
narrow the rows of a prefix of the vocabulary (WMD_DROPIN_HOST_SHARE of V,
by default a share with at least 4 host threads) to FP32 and copy them,
while the GPU reads, above the prefix, only the rows of the words that occur
in the target matrix or in r, in FP64 from the pinned buffer itself;
pageable embeddings are narrowed on the host whole (share > 0) or copied
whole (share 0).  The results must be bit-identical on every path (one
FP64 -> FP32 rounding, one norm summation order, and the solve never touches
any other row), and ``wmd_dropin_h2d_bytes`` must count exactly the bytes
that crossed the bus.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bytes(V, d, N, nnz, rows):
    # target matrix (col_ptr, rows, vals) + length order + r + FP64 rows
    return (N + 1) * 8 + nnz * 16 + N * 4 + V * 8 + rows * d * 8


def _bytes_split(V, d, N, nnz, host_rows, dev_rows):
    # the same with the host-narrowed FP32 prefix rows and the FP64 rows the
    # GPU reads itself
    return (N + 1) * 8 + nnz * 16 + N * 4 + V * 8 + host_rows * d * 4 + dev_rows * d * 8


@pytest.mark.parametrize("params", [
    (3000, 300, 60, 32, 8, 128, 50, 70),           # v_r = 32
    (2000, 7, 80, 20, 4, 40, 30, 71, 10.0, 15, 5),  # d = 7, empty documents
])
def test_dropin_moves_only_needed_rows(wmd, synth, params, monkeypatch):
    p = synth.case(*params)
    V, d = p.vecs.shape
    N = p.col_ptr.size - 1
    nnz = p.row_inds.size
    vecs = np.ascontiguousarray(p.vecs, np.float64)
    args = (p.col_ptr, p.row_inds, p.vals)
    needed = np.union1d(np.unique(p.row_inds), np.flatnonzero(p.r))
    assert needed.size < V
    pin = torch.from_numpy(vecs.copy()).pin_memory()
    for variant, lam in (("fused", -p.lam), ("nonfused", p.lam)):
        monkeypatch.setenv("WMD_DROPIN_HOST_SHARE", "0")
        ref = wmd.sinkhorn_wmd_csc(p.r, vecs, *args, lam, p.max_iter, variant)
        assert wmd.dropin_h2d_bytes() == _bytes(V, d, N, nnz, V)  # whole copy
        for share in (0.0, 0.25, 0.5, 1.0):
            monkeypatch.setenv("WMD_DROPIN_HOST_SHARE", str(share))
            got = wmd.sinkhorn_wmd_csc(p.r, pin.numpy(), *args, lam, p.max_iter, variant)
            np.testing.assert_array_equal(got, ref)
            wh = int(share * V + 0.5)  # host prefix; needed rows above it
            above = int((needed >= wh).sum())
            assert wmd.dropin_h2d_bytes() == _bytes_split(V, d, N, nnz, wh, above)
            if share > 0:  # pageable: every row narrowed on the host
                got = wmd.sinkhorn_wmd_csc(p.r, vecs, *args, lam, p.max_iter, variant)
                np.testing.assert_array_equal(got, ref)
                assert wmd.dropin_h2d_bytes() == _bytes_split(V, d, N, nnz, V, 0)
        monkeypatch.delenv("WMD_DROPIN_HOST_SHARE")


def test_pinned_view_at_an_offset_and_csr_drop_in(wmd, synth, monkeypatch):
    """A view into a larger pinned buffer is read in place as well; the CSR
    drop-in (the reference's own call shape) takes the same path."""
    monkeypatch.setenv("WMD_DROPIN_HOST_SHARE", "0")
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
    assert wmd.dropin_h2d_bytes() == _bytes_split(V, d, N, p.row_inds.size, 0, used.size)
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
    # the low half of the vocabulary narrowed on the host: the same scores
    monkeypatch.setenv("WMD_DROPIN_HOST_SHARE", "0.5")
    np.testing.assert_array_equal(wmd.sinkhorn_wmd_fused(p.r, view, *csr_args), csr_pinned)
