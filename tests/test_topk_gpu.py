"""GPU: top-k nearest documents, bit-exact against numpy's stable argsort
(ascending, ties by index, NaN last) of the same scores."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _expected(scores, k):
    s = np.where(scores == 0.0, 0.0, scores)  # -0.0 ties with +0.0
    order = np.argsort(s, kind="stable")[:k]
    return order.astype(np.uint32), scores[order]


@pytest.mark.parametrize("n,k", [(1, 1), (5, 10), (2047, 7), (2048, 100),
                                 (2049, 1024), (50_000, 1), (50_000, 100),
                                 (300_000, 333)])
def test_topk_device_matches_stable_argsort(wmd, n, k):
    import torch
    rng = np.random.default_rng(n + k)
    # few distinct values -> many ties; plus signed zeros, infinities, NaN
    s = np.round(rng.normal(size=n), 1)
    if n > 10:
        s[rng.integers(0, n, 5)] = -0.0
        s[rng.integers(0, n, 3)] = np.inf
        s[rng.integers(0, n, 3)] = -np.inf
        s[rng.integers(0, n, 7)] = np.nan
    eng = wmd.Engine()
    sd = torch.from_numpy(s).cuda()
    idx = torch.empty(k, dtype=torch.int32, device="cuda")
    val = torch.empty(k, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the engine runs on its own stream
    eng.topk_device(sd.data_ptr(), n, k, idx.data_ptr(), val.data_ptr())
    eng.check()
    got_i = idx.cpu().numpy().view(np.uint32)
    got_v = val.cpu().numpy()
    exp_i, exp_v = _expected(s, k)
    m = min(n, k)
    np.testing.assert_array_equal(got_i[:m], exp_i)
    np.testing.assert_array_equal(np.nan_to_num(got_v[:m], nan=7.0),
                                  np.nan_to_num(np.where(exp_v == 0, 0.0, exp_v), nan=7.0))
    if k > n:
        assert np.all(got_i[n:] == np.uint32(0xFFFFFFFF))
    eng.close()


def test_query_topk_on_scores(wmd, synth):
    p = synth.case(3000, 300, 2500, 32, 8, 100, 40, 400, empty_every=97)
    # every document twice: equal scores, so ties are broken by index
    lens = np.diff(p.col_ptr)
    cp = np.concatenate([[0], np.cumsum(np.concatenate([lens, lens]))])
    rows = np.concatenate([p.row_inds, p.row_inds])
    vals = np.concatenate([p.vals, p.vals])
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(cp, rows, vals)
    scores = eng.query(p.r, p.lam, p.max_iter)
    for k in (1, 16, 500):
        idx, val = eng.query_topk(p.r, p.lam, p.max_iter, k)
        exp_i, exp_v = _expected(scores, k)
        np.testing.assert_array_equal(idx, exp_i)
        np.testing.assert_array_equal(np.isnan(val), np.isnan(exp_v))
        np.testing.assert_array_equal(val[~np.isnan(val)], exp_v[~np.isnan(exp_v)])
    eng.close()


def test_topk_rejects_bad_k(wmd, synth):
    p = synth.case(500, 300, 20, 8, 4, 20, 10, 5)
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    for k in (0, 1025):
        with pytest.raises(wmd.WMDError) as e:
            eng.query_topk(p.r, p.lam, p.max_iter, k)
        assert e.value.name == "WMD_ERR_INVALID_ARG"
    idx, val = eng.query_topk(p.r, p.lam, p.max_iter, 20)
    assert sorted(idx.tolist()) == list(range(20))
    eng.close()
