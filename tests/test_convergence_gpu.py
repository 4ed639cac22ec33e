"""GPU: per-document convergence stopping (tolerance on the marginal
residual) against the oracle's converged FP64 mode, which applies the same
stopping rule (iterate until sum_i |u_i (K v)_i - r_i| <= tol, then form the
WMD with the updated scalings)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tol", [1e-3, 1e-5])
def test_converged_solve_matches_fp64_oracle(wmd, synth, oracle_mod, tol):
    p = synth.case(4000, 300, 300, 32, 8, 200, 60, 300)
    cap = 3000
    ref, ref_it, ref_res, _ = oracle_mod.sinkhorn_converged(
        p.r, p.vecs.astype(np.float64), p.col_ptr, p.row_inds, p.vals, p.lam,
        tol=tol, max_iter_cap=cap)
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.set_tolerance(tol)
    got = eng.query(p.r, p.lam, cap)
    it = eng.last_iterations()
    # Iteration counts agree except where FP32 rounding moves the residual
    # across the threshold by one update.
    assert np.mean(np.abs(it - ref_it) <= 1) >= 0.97
    same = it == ref_it
    assert rel_err(got[same], ref[same]).max() <= 2e-5
    # Documents stopping one update apart still agree to the tolerance scale.
    assert rel_err(got, ref).max() <= 50 * tol
    # tol = 0 restores the fixed count of the reference
    eng.set_tolerance(0.0)
    fixed = eng.query(p.r, p.lam, 15)
    assert np.all(eng.last_iterations() == 15)
    ref15 = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                                p.row_inds, p.vals, p.lam, 15)
    assert rel_err(fixed, ref15).max() <= 1e-5
    eng.close()


@pytest.mark.parametrize("vr,prec", [(32, "fp32"), (200, "bf16")])
def test_over_relaxation_same_fixed_point_fewer_updates(wmd, synth, oracle_mod, vr, prec):
    """omega > 1 stops (residual <= 1e-5) within 1e-4 of the converged FP64
    oracle like omega = 1, in fewer updates on average."""
    p = synth.case(4000, 300, 300, vr, 8, 200, 60, 500 + vr)
    conv = oracle_mod.sinkhorn_converged(p.r, p.vecs.astype(np.float64), p.col_ptr,
                                         p.row_inds, p.vals, p.lam, tol=1e-10,
                                         max_iter_cap=50000)[0]
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.set_solve_precision(prec)
    eng.set_tolerance(1e-5)
    its = {}
    for omega in (1.0, 1.6):
        eng.set_relaxation(omega)
        got = eng.query(p.r, p.lam, 5000)
        it = eng.last_iterations()
        done = it < 5000
        assert done.mean() > 0.95
        assert rel_err(got[done], conv[done]).max() <= 1e-4
        its[omega] = it.mean()
    assert its[1.6] < its[1.0], its
    with pytest.raises(wmd.WMDError):
        eng.set_relaxation(2.0)
    eng.close()


@pytest.mark.parametrize("vr,prec", [(32, "fp32"), (300, "bf16"), (128, "bf16")])
def test_over_relaxation_guard_keeps_aggressive_omega_safe(wmd, synth, oracle_mod, vr, prec):
    """Both half-steps relaxed at omega = 1.95, where the plain relaxed
    iteration diverges on wide sources: the per-document guard steps omega
    back, every finished document stays within 1e-4 of the converged FP64
    oracle.  Without a tolerance (a fixed update count) relaxation does not
    apply: the results are the reference iteration's, bit for bit."""
    p = synth.case(4000, 300, 200, vr, 8, 200, 60, 700 + vr)
    conv = oracle_mod.sinkhorn_converged(p.r, p.vecs.astype(np.float64), p.col_ptr,
                                         p.row_inds, p.vals, p.lam, tol=1e-10,
                                         max_iter_cap=50000)[0]
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.set_solve_precision(prec)
    eng.set_tolerance(1e-5)
    eng.set_relaxation(1.95)
    got = eng.query(p.r, p.lam, 5000)
    it = eng.last_iterations()
    done = it < 5000
    assert done.mean() > 0.9
    assert np.all(np.isfinite(got))
    assert rel_err(got[done], conv[done]).max() <= 1e-4
    eng.set_tolerance(0.0)
    fixed = eng.query(p.r, p.lam, 40)
    eng.set_relaxation(1.0)
    np.testing.assert_array_equal(fixed, eng.query(p.r, p.lam, 40))
    eng.close()
