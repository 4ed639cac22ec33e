"""GPU: batched queries (many sources, one call) against single-source
queries and the oracle."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(synth):
    V, N = 5000, 300
    cdf = synth.zipf_cdf(V)
    vecs = synth.embeddings(V, 300, 60, seed=40)
    cp, ri, vv = synth.targets(V, N, 8, 160, seed=41, cdf=cdf)
    vrs = [1, 5, 17, 32, 33, 64, 100, 300, 0]
    rs = [synth.source_doc(V, v, seed=50 + k, cdf=cdf) if v else np.zeros(V)
          for k, v in enumerate(vrs)]
    return vecs, cp, ri, vv, rs


@pytest.mark.parametrize("mode", ["fp32", "fp16", "tf32x3"])
def test_batch_equals_single_queries(wmd, oracle_mod, problem, mode):
    vecs, cp, ri, vv, rs = problem
    eng = wmd.Engine()
    eng.set_cdist_mode(mode)
    eng.set_embeddings(vecs)
    eng.set_targets(cp, ri, vv)
    out, iters = eng.query_batch(rs, 10.0, 15, want_iters=True)
    assert out.shape == (len(rs), cp.size - 1)
    assert np.all(iters == 15)
    for k, r in enumerate(rs):
        single = eng.query(r, 10.0, 15)
        np.testing.assert_array_equal(out[k], single)
        if mode in ("fp32", "tf32x3"):
            ref = oracle_mod.sinkhorn(r, vecs.astype(np.float64), cp, ri, vv, 10.0, 15)
            np.testing.assert_array_equal(np.isnan(out[k]), np.isnan(ref))
            assert rel_err(out[k], ref).max() <= 1e-5
    np.testing.assert_array_equal(out[-1], np.zeros(cp.size - 1))  # empty source
    eng.close()


def test_batch_sparse_input_and_validation(wmd, problem):
    vecs, cp, ri, vv, rs = problem
    eng = wmd.Engine()
    eng.set_embeddings(vecs)
    eng.set_targets(cp, ri, vv)
    r = rs[3]
    ids = np.nonzero(r)[0]
    sparse = (ids[::-1].copy(), r[ids][::-1].copy())  # unsorted: the wrapper sorts
    out = eng.query_batch([sparse, r], 10.0, 15)
    np.testing.assert_array_equal(out[0], out[1])
    bad = (np.array([1, 1, 2]), np.array([0.3, 0.3, 0.4]))  # duplicate id
    with pytest.raises(wmd.WMDError) as e:
        eng.query_batch([bad], 10.0, 15)
    assert e.value.name == "WMD_ERR_INVALID_INPUT"
    eng.close()
