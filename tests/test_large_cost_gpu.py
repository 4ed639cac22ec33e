"""GPU: costs whose lambda * M underflows FP32.

The reference keeps K = exp(lamda M) in FP64 (sinkhorn_wmd_fused.cpp:217),
finite to lambda M ~ 708; FP32 underflows near 87.  With the embeddings
scaled by alpha (distances scale with it), lambda = 10 spans lambda M up to
~32 alpha: 96 (alpha 3), 191 (alpha 6) and 319 (alpha 10).  The engine then
keeps each vocabulary row scaled to its largest entry and re-solves in FP64
the documents the FP32 panel still cannot carry; every document must come out
finite where the FP64 oracle (pinned bit-exact to the reference) is, and
agree with it.

Tolerance: 1e-4 relative.  At these sizes M itself is ~20-30 and its FP32
rounding alone moves K by lambda * ulp(M) ~ 2e-5 relative, so the plain
path's 1e-5 does not apply; alpha = 1 (lambda M <= 32) keeps 1e-5 (1e-4 for
the BF16 panel, its usual bar).  In the row-scaled form the engine keeps the
FP32 panel even when the BF16 one is requested.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _case(synth, alpha, v_r, seed):
    p = synth.case(3000, 300, 200, v_r, 8, 128, 50, seed)
    p.vecs = (p.vecs * np.float32(alpha)).astype(np.float32)
    return p


def _oracle(oracle_mod, p, max_iter=None):
    return oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                               p.row_inds, p.vals, p.lam,
                               p.max_iter if max_iter is None else max_iter)


@pytest.mark.parametrize("alpha", [1.0, 3.0, 6.0, 10.0])
@pytest.mark.parametrize("v_r", [32, 200])
@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_large_lambda_m_vs_oracle(wmd, synth, oracle_mod, alpha, v_r, prec):
    if prec == "bf16" and v_r <= 64:
        pytest.skip("the BF16 panel serves 64 < v_r <= 512 only")
    p = _case(synth, alpha, v_r, 77 + v_r)
    ref = _oracle(oracle_mod, p)
    assert np.isfinite(ref).all()
    eng = wmd.Engine(0)
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.set_cdist_mode("tf32x3")
    eng.set_solve_precision(prec)
    got = eng.query(p.r, p.lam, p.max_iter)
    eng.close()
    assert np.isfinite(got).all(), f"{(~np.isfinite(got)).sum()} documents not finite"
    # BF16 panel (alpha = 1): its own 1e-4 bar; alpha >= 3 runs the FP32 panel
    tol = 1e-5 if (alpha == 1.0 and prec == "fp32") else 1e-4
    err = rel_err(got, ref)
    assert err.max() <= tol, f"max rel err {err.max():.3e}"


@pytest.mark.parametrize("mode", ["fp32", "tf32x3", "f16x3", "bf16"])
def test_large_lambda_m_cost_panels_and_batch(wmd, synth, oracle_mod, mode):
    """Every cost-panel form and the batched path take the row-scaled form
    (the split-FP16 form for the single query; its batches run split-TF32)."""
    p = _case(synth, 6.0, 40, 91)
    srcs = [p.r] + [synth.source_doc(p.V, v, seed=400 + v) for v in (12, 90)]
    refs = [oracle_mod.sinkhorn(r, p.vecs.astype(np.float64), p.col_ptr, p.row_inds,
                                p.vals, p.lam, p.max_iter) for r in srcs]
    eng = wmd.Engine(0)
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.set_cdist_mode(mode)
    got = eng.query_batch(srcs, p.lam, p.max_iter)
    one = eng.query(srcs[1], p.lam, p.max_iter)
    eng.close()
    # BF16 operands: M itself is off by ~1e-4 x alpha there
    tol = 5e-3 if mode == "bf16" else 1e-4
    for g, r in zip(got, refs):
        assert np.isfinite(g).all()
        assert rel_err(g, r).max() <= tol
    assert rel_err(one, refs[1]).max() <= tol


def test_large_lambda_m_dropin_and_converged(wmd, synth, oracle_mod):
    """The drop-in call, and the per-document stopping rule on the
    row-scaled panel against the converged FP64 oracle."""
    p = _case(synth, 6.0, 32, 93)
    ref = _oracle(oracle_mod, p)
    got = wmd.sinkhorn_wmd_csc(p.r, p.vecs.astype(np.float64), p.col_ptr,
                               p.row_inds, p.vals, -p.lam, p.max_iter, "fused")
    assert np.isfinite(got).all()
    assert rel_err(got, ref).max() <= 1e-4
    m = 50  # documents checked against the converged oracle
    cp = p.col_ptr[:m + 1]
    conv, _, _, _ = oracle_mod.sinkhorn_converged(
        p.r, p.vecs.astype(np.float64), cp, p.row_inds[:cp[-1]], p.vals[:cp[-1]],
        p.lam, tol=1e-9, max_iter_cap=100000)
    eng = wmd.Engine(0)
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.set_tolerance(1e-5)
    c = eng.query(p.r, p.lam, 20000)
    it = eng.last_iterations()
    eng.close()
    done = it[:m] < 20000
    assert done.mean() > 0.9
    assert rel_err(c[:m][done], conv[done]).max() <= 1e-4
