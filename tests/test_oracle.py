"""CPU: the oracle restatement pinned to the reference's own outputs.

golden.json was produced by running the reference's solvers (compiled from
its sources) and its Python main.py; these tests need neither at run time.
When oracle/_ref/ exists (the reference was compiled here) the live
reference is compared too.
"""
import numpy as np
import pytest

from cases import SYNTH_CASES
from conftest import rel_err


def _sample(golden):
    s = golden["sample_d3"]
    rows, cols, w = s["edges"]
    return s, np.array(rows), np.array(cols), np.array(w, float)


def test_sample_known_answers_match_reference_readme_values(golden):
    # The d=3 "small input" of the reference README, lamda=-1, 15 iterations.
    out = golden["sample_d3"]["outputs"]
    np.testing.assert_allclose(
        out["fused_lam1"],
        [0.88632517, 0.343080145, 0.340746603, 0.659569734, 0.869842081],
        rtol=6e-9)  # the reference prints 9 significant digits (fused:621)
    np.testing.assert_allclose(
        out["nonfused_shipped_sign"],
        [1.19635575, 0.343080145, 0.340746603, 0.708083763, 0.99402085],
        rtol=6e-9)  # the reference prints 9 significant digits (fused:621)
    # fused(-lam) == nonfused(+lam) == main.py(lamb=-lam)
    for lam in ("1", "10"):
        np.testing.assert_array_equal(out[f"fused_lam{lam}"], out[f"nonfused_lam{lam}"])
        assert rel_err(out[f"mainpy_lam{lam}"], out[f"fused_lam{lam}"]).max() < 1e-12


@pytest.mark.parametrize("lam", [1.0, 10.0])
def test_oracle_sample_bit_exact(golden, oracle_mod, lam):
    s, rows, cols, w = _sample(golden)
    col_ptr, ri, rv = oracle_mod.counting_sort(s["N"], cols, rows, w)
    got = oracle_mod.sinkhorn(np.array(s["r"]), np.array(s["vecs"]), col_ptr,
                              ri, rv, lam, s["max_iter"], nthreads=1)
    np.testing.assert_array_equal(got, s["outputs"][f"fused_lam{lam:g}"])


@pytest.mark.parametrize("name", sorted(SYNTH_CASES))
def test_oracle_synthetic_vs_reference_golden(golden, synth, oracle_mod, name):
    g = golden["synthetic"][name]
    p = synth.case(*g["params"])
    assert synth.digest(p) == g["digest"], "synthetic generator changed"
    got = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                              p.row_inds, p.vals, p.lam, p.max_iter, nthreads=1)
    ref = np.array(g["fused"])
    # One thread on both sides: the same FP64 operation order -> bit-exact.
    np.testing.assert_array_equal(got, ref)
    if "mainpy" in g:
        assert rel_err(g["mainpy"], ref).max() < 1e-9


def test_oracle_threads_do_not_change_results(synth, oracle_mod):
    p = synth.case(*SYNTH_CASES["vr32_basic"][:6], 50, 10)
    a = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                            p.row_inds, p.vals, 10.0, 15, nthreads=1)
    b = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                            p.row_inds, p.vals, 10.0, 15, nthreads=4)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("variant", ["fused", "nonfused"])
def test_live_reference_vs_oracle(synth, oracle_mod, variant):
    if not oracle_mod.reference_available(variant):
        pytest.skip("reference not compiled here (oracle/_ref absent)")
    from oracle import oracle as O
    p = synth.case(*SYNTH_CASES["vr33"])
    csr = oracle_mod.csr_from_csc(p.V, p.N, p.col_ptr, p.row_inds, p.vals)
    ref = O.reference_sinkhorn(p.r, p.vecs.astype(np.float64), *csr, p.N,
                               p.lam, p.max_iter, variant, 4)
    got = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                              p.row_inds, p.vals, p.lam, p.max_iter, nthreads=4)
    # Multi-threaded reference scatters with omp atomic (fused:284): the
    # summation order varies, so compare to a few ulps.
    assert rel_err(got, ref).max() < 1e-12


def test_converged_mode_reaches_tolerance_and_fixed_point(synth, oracle_mod):
    p = synth.case(*SYNTH_CASES["vr17_lambda1"])
    w, iters, res, u = oracle_mod.sinkhorn_converged(
        p.r, p.vecs.astype(np.float64), p.col_ptr, p.row_inds, p.vals, p.lam,
        tol=1e-10, max_iter_cap=20000, want_u=True)
    assert np.all(res <= 1e-10)
    # Running the fixed-count solve for each document's iteration count
    # reproduces the converged value.
    k = int(np.median(iters))
    sel = np.nonzero(iters == k)[0][:5]
    for j in sel:
        cp = np.array([0, p.col_ptr[j + 1] - p.col_ptr[j]])
        seg = slice(p.col_ptr[j], p.col_ptr[j + 1])
        one = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), cp,
                                  p.row_inds[seg], p.vals[seg], p.lam, k)
        assert rel_err(one, w[j:j + 1]).max() < 1e-13


def test_counting_sort_stable_and_transposes(oracle_mod):
    rng = np.random.default_rng(0)
    V, N, nnz = 50, 30, 400
    rows = rng.integers(0, V, nnz)
    cols = rng.integers(0, N, nnz)
    w = rng.integers(1, 9, nnz).astype(np.float64)
    ptr, oc, ow = oracle_mod.counting_sort(V, rows, cols, w)
    # stable: within a row, original order preserved
    for i in range(V):
        idx = np.nonzero(rows == i)[0]
        np.testing.assert_array_equal(oc[ptr[i]:ptr[i + 1]], cols[idx])
        np.testing.assert_array_equal(ow[ptr[i]:ptr[i + 1]], w[idx])
    cp, rr, vv = oracle_mod.csc_from_csr(V, N, ptr, oc, ow)
    from scipy import sparse
    A = sparse.csr_matrix((ow, oc, ptr), shape=(V, N)).toarray()
    B = sparse.csc_matrix((vv, rr, cp), shape=(V, N)).toarray()
    np.testing.assert_array_equal(A, B)
    for j in range(N):
        assert np.all(np.diff(rr[cp[j]:cp[j + 1]].astype(np.int64)) >= 0)
