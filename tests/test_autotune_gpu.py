"""GPU: the launch-shape autotuner of the plain warp solve.  The first query
of each lane layout times every candidate shape on the handle's own panel
and target set and keeps the fastest; every candidate runs the same
per-document arithmetic, so the scores do not depend on the choice."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_warp_solve_shape_is_tuned_and_results_unchanged(wmd, synth, oracle_mod):
    p = synth.case(4000, 300, 400, 32, 8, 200, 50, 61)
    q = synth.source_doc(p.V, 90, seed=62)
    eng = wmd.Engine(0)
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    got = eng.query(p.r, p.lam, p.max_iter)
    got_w = eng.query(q, p.lam, p.max_iter)
    ch = eng.solve_shape_choices()
    assert 32 in ch and 128 in ch, ch
    assert all(v != "build-time default" for v in ch.values()), ch
    ref = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr, p.row_inds,
                              p.vals, p.lam, p.max_iter)
    assert rel_err(got, ref).max() <= 1e-5
    # tuning off: the build-time default shape, bit-identical scores
    eng.set_autotune(False)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)  # forgets the choices
    again = eng.query(p.r, p.lam, p.max_iter)
    again_w = eng.query(q, p.lam, p.max_iter)
    assert eng.solve_shape_choices() == {}
    np.testing.assert_array_equal(got, again)
    np.testing.assert_array_equal(got_w, again_w)
    eng.close()
