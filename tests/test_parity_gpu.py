"""GPU parity: the CUDA path through the C ABI against the reference's FP64
output (golden fixtures) and the oracle.

Tolerance: the plain path computes the cost panel and the Sinkhorn
iterations in FP32 (FP64 only in the final per-document reduction), so it is
held to 1e-5 relative error per document against the reference's FP64
result, the bar the plain path is specified to.  Documents the reference
scores as NaN (empty documents: u = 1/0 times x = 0, fused:382-393) must be
NaN here too.
"""
import numpy as np
import pytest

from cases import SYNTH_CASES
from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _problem(synth, golden, name):
    g = golden["synthetic"][name]
    p = synth.case(*g["params"])
    assert synth.digest(p) == g["digest"], "synthetic generator changed"
    return p, np.array(g["fused"])


def _check(got, ref, tol=TOL):
    got, ref = np.asarray(got), np.asarray(ref)
    assert got.shape == ref.shape
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    err = rel_err(got, ref)
    assert err.max() <= tol, f"max rel err {err.max():.3e} at {int(err.argmax())}"
    return err.max()


@pytest.mark.parametrize("name", sorted(SYNTH_CASES))
@pytest.mark.parametrize("variant", ["fused", "nonfused"])
def test_synthetic_csc_parity(wmd, synth, golden, name, variant):
    p, ref = _problem(synth, golden, name)
    lamda = -p.lam if variant == "fused" else p.lam
    got = wmd.sinkhorn_wmd_csc(p.r, p.vecs.astype(np.float64), p.col_ptr,
                               p.row_inds, p.vals, lamda, p.max_iter, variant)
    _check(got, ref)


@pytest.mark.parametrize("name", ["vr32_basic", "empty_docs", "vr100", "d7_unaligned"])
def test_synthetic_csr_dropin_parity(wmd, synth, golden, oracle_mod, name):
    p, ref = _problem(synth, golden, name)
    row_ptr, ci, cv = oracle_mod.csr_from_csc(p.V, p.N, p.col_ptr, p.row_inds, p.vals)
    got = wmd.sinkhorn_wmd_fused(p.r, p.vecs.astype(np.float64), -p.lam,
                                 p.max_iter, row_ptr, ci, cv, p.N)
    _check(got, ref)
    got2 = wmd.sinkhorn_wmd_nonfused(p.r, p.vecs.astype(np.float64), p.lam,
                                     p.max_iter, row_ptr, ci, cv, p.N)
    _check(got2, ref)


@pytest.mark.parametrize("key,lamda,variant", [
    ("fused_lam1", -1.0, "fused"), ("fused_lam10", -10.0, "fused"),
    ("nonfused_lam10", 10.0, "nonfused"),
    ("nonfused_shipped_sign", -1.0, "nonfused")])
def test_sample_d3_known_answers(wmd, golden, oracle_mod, key, lamda, variant):
    s = golden["sample_d3"]
    rows, cols, w = (np.array(a) for a in s["edges"])
    row_ptr, ci, cv = oracle_mod.counting_sort(s["N"], rows, cols, w)
    fn = wmd.sinkhorn_wmd_fused if variant == "fused" else wmd.sinkhorn_wmd_nonfused
    got = fn(np.array(s["r"]), np.array(s["vecs"]), lamda, s["max_iter"],
             row_ptr, ci, cv, s["N"])
    _check(got, s["outputs"][key])


def test_mainpy_mirror(wmd, synth, golden):
    from scipy import sparse
    g = golden["synthetic"]["vr32_basic"]
    p = synth.case(*g["params"])
    c = sparse.csc_matrix((p.vals, p.row_inds, p.col_ptr), shape=(p.V, p.N)).tocsr()
    got = wmd.sinkhorn_wmd(p.r, c, p.vecs.astype(np.float64), -p.lam, p.max_iter)
    assert got.shape == (1, p.N)
    _check(np.asarray(got).ravel(), g["mainpy"])


def test_empty_source_gives_zero(wmd, synth):
    p = synth.case(500, 300, 20, 8, 4, 20, 10, 5)
    got = wmd.sinkhorn_wmd_csc(np.zeros(p.V), p.vecs, p.col_ptr, p.row_inds,
                               p.vals, -10.0, 15)
    # v_r = 0: the reference sums over no source words (fused:382-393).
    np.testing.assert_array_equal(got, np.zeros(p.N))


def test_invalid_inputs_return_status(wmd, synth):
    p = synth.case(500, 300, 20, 8, 4, 20, 10, 5)
    bad_rows = p.row_inds.copy()
    bad_rows[3] = p.V  # word index out of range
    with pytest.raises(wmd.WMDError) as e:
        wmd.sinkhorn_wmd_csc(p.r, p.vecs, p.col_ptr, bad_rows, p.vals, -10.0, 15)
    assert e.value.name == "WMD_ERR_INVALID_INPUT"
    neg = p.r.copy()
    neg[np.nonzero(neg)[0][0]] = -0.5  # the reference driver rejects r < 0
    with pytest.raises(wmd.WMDError) as e:
        wmd.sinkhorn_wmd_csc(neg, p.vecs, p.col_ptr, p.row_inds, p.vals, -10.0, 15)
    assert e.value.name == "WMD_ERR_INVALID_INPUT"
    zval = p.vals.copy()
    zval[0] = 0.0  # the reference driver rejects weights <= 0
    with pytest.raises(wmd.WMDError) as e:
        wmd.sinkhorn_wmd_csc(p.r, p.vecs, p.col_ptr, p.row_inds, zval, -10.0, 15)
    assert e.value.name == "WMD_ERR_INVALID_INPUT"
    cp = p.col_ptr.copy()
    cp[5], cp[6] = cp[6], cp[5]
    with pytest.raises(wmd.WMDError):
        wmd.sinkhorn_wmd_csc(p.r, p.vecs, cp, p.row_inds, p.vals, -10.0, 15)
    # the library stays usable after rejected calls
    ok = wmd.sinkhorn_wmd_csc(p.r, p.vecs, p.col_ptr, p.row_inds, p.vals, -10.0, 15)
    assert np.all(np.isfinite(ok))


@pytest.fixture(scope="module")
def full(synth, oracle_mod):
    """The single-source workload at its full size: V=1e5, d=300, v_r=32,
    N=5000, nnz ~ U[8,256], lambda=10, 15 iterations."""
    p = synth.single_source()
    ref = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                              p.row_inds, p.vals, p.lam, p.max_iter)
    return p, ref


def test_full_size_parity_and_determinism(wmd, full):
    p, ref = full
    a = wmd.sinkhorn_wmd_csc(p.r, p.vecs.astype(np.float64), p.col_ptr,
                             p.row_inds, p.vals, -p.lam, p.max_iter)
    _check(a, ref)
    b = wmd.sinkhorn_wmd_csc(p.r, p.vecs.astype(np.float64), p.col_ptr,
                             p.row_inds, p.vals, -p.lam, p.max_iter)
    np.testing.assert_array_equal(a, b)  # no atomics: bitwise reproducible


def test_full_size_document_independence(wmd, full):
    """Size-independent properties at full size: permuting the documents
    permutes the scores bit-for-bit, and any subset scores identically."""
    p, ref = full
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    base = eng.query(p.r, p.lam, p.max_iter)
    _check(base, ref)
    rng = np.random.default_rng(3)
    perm = rng.permutation(p.N)
    lens = np.diff(p.col_ptr)[perm]
    cp = np.zeros(p.N + 1, np.int64)
    cp[1:] = np.cumsum(lens)
    rows = np.concatenate([p.row_inds[p.col_ptr[j]:p.col_ptr[j + 1]] for j in perm])
    vals = np.concatenate([p.vals[p.col_ptr[j]:p.col_ptr[j + 1]] for j in perm])
    eng.set_targets(cp, rows, vals)
    permuted = eng.query(p.r, p.lam, p.max_iter)
    np.testing.assert_array_equal(permuted, base[perm])
    eng.close()


def test_device_resident_query_matches_host_query(wmd, full):
    import torch
    p, ref = full
    eng = wmd.Engine()
    eng.set_embeddings(torch.from_numpy(p.vecs).cuda())
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    r = torch.from_numpy(p.r).cuda()
    out = torch.empty(p.N, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    eng.query_device(r.data_ptr(), 64, p.lam, p.max_iter, out.data_ptr())
    eng.check()
    got = out.cpu().numpy()
    _check(got, ref)
    assert eng.launch_count >= 3
    # vr_cap smaller than the true v_r is reported, not silently truncated
    eng.query_device(r.data_ptr(), 8, p.lam, p.max_iter, out.data_ptr())
    with pytest.raises(wmd.WMDError):
        eng.check()
    eng.close()


@pytest.mark.parametrize("lam", [0.0, 0.5, -1.0])
def test_lambda_edge_values_vs_oracle(wmd, synth, oracle_mod, lam):
    """lambda = 0 (K = 1: the solve reads the stored K.*M panel instead of
    recovering M from K) and the reference's shipped nonfused sign
    (lambda = -1: K = exp(+M))."""
    p = synth.case(1500, 300, 80, 24, 8, 60, 30, 210)
    ref = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                              p.row_inds, p.vals, lam, 15, nthreads=1)
    got = wmd.sinkhorn_wmd_csc(p.r, p.vecs.astype(np.float64), p.col_ptr,
                               p.row_inds, p.vals, -lam, 15, "fused")
    _check(got, ref)


def test_device_query_graph_replay(wmd, synth, oracle_mod):
    """Repeated device queries are captured once into a CUDA graph and
    replayed; a query that grows the working buffers in between, or a new
    target set, must never replay a graph holding stale addresses."""
    import torch
    p = synth.case(3000, 300, 400, 32, 8, 200, 50, 220)
    ref = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                              p.row_inds, p.vals, p.lam, p.max_iter)
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    r = torch.from_numpy(p.r).cuda()
    outs = []
    for cap in (32, 32, 32, 32, 200, 32, 32):
        out = torch.full((p.N,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        eng.query_device(r.data_ptr(), cap, p.lam, p.max_iter, out.data_ptr())
        eng.check()
        outs.append(out.cpu().numpy())
        del out
    for o in outs:
        _check(o, ref)
    np.testing.assert_array_equal(outs[0], outs[3])  # eager == replayed
    np.testing.assert_array_equal(outs[0], outs[6])
    # new target set (half the documents): same engine, same pointers
    half = p.N // 2
    cp = p.col_ptr[:half + 1]
    eng.set_targets(cp, p.row_inds[:cp[-1]], p.vals[:cp[-1]])
    out = torch.empty(half, dtype=torch.float64, device="cuda")
    for _ in range(3):
        eng.query_device(r.data_ptr(), 32, p.lam, p.max_iter, out.data_ptr())
        eng.check()
        np.testing.assert_array_equal(out.cpu().numpy(), outs[0][:half])
    eng.close()
