"""GPU: the word-major solve order (the reference's own traversal,
sinkhorn_wmd_fused.cpp:249-292) against the FP64 oracle and the
document-major solve.  Its x is summed with atomics, so the order of the
FP32 additions varies; the bar is the plain path's 1e-5."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _engine(wmd, p):
    eng = wmd.Engine(0)
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    return eng


@pytest.mark.parametrize("v_r", [1, 3, 32, 33, 200, 512])
def test_word_major_vs_oracle(wmd, synth, oracle_mod, v_r):
    p = synth.case(3000, 300, 150, v_r, 1, 180, 50, 200 + v_r, empty_every=23)
    ref = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr, p.row_inds,
                              p.vals, p.lam, p.max_iter)
    eng = _engine(wmd, p)
    doc = eng.query(p.r, p.lam, p.max_iter)
    eng.set_solve_order("word")
    got = eng.query(p.r, p.lam, p.max_iter)
    got2 = eng.query(p.r, p.lam, p.max_iter)  # graph replay
    eng.close()
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    assert rel_err(got, ref).max() <= TOL
    assert rel_err(got2, ref).max() <= TOL
    assert rel_err(got, doc).max() <= TOL


def test_word_major_row_scaled_and_limits(wmd, synth, oracle_mod):
    p = synth.case(3000, 300, 150, 24, 8, 120, 50, 301)
    p.vecs = (p.vecs * np.float32(6.0)).astype(np.float32)  # lambda M up to ~190
    ref = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr, p.row_inds,
                              p.vals, p.lam, p.max_iter)
    eng = _engine(wmd, p)
    eng.set_solve_order("word")
    got = eng.query(p.r, p.lam, p.max_iter)
    assert np.isfinite(got).all()
    assert rel_err(got, ref).max() <= 1e-4
    eng.set_tolerance(1e-4)  # per-document stopping: document-major only
    with pytest.raises(wmd.WMDError):
        eng.query(p.r, p.lam, 100)
    eng.set_tolerance(0.0)
    with pytest.raises(wmd.WMDError):
        eng.query_batch([p.r], p.lam, p.max_iter)
    eng.close()
