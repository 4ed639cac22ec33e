"""GPU: the learned warm start against its CPU oracle.

* gradients of the hand-written forward/backward kernels vs the float64
  oracle (FP32 kernels: relative 1e-3 of the largest gradient entry);
* labels (FP64 converged solve on the GPU) vs the FP64 oracle's converged
  scalings, and the raw features vs features computed from the embeddings;
* the fused tensor-core inference (BF16 layer 2, tanh.approx GELU) vs the
  oracle's forward on the same features (absolute 0.05 in log u);
* end to end: a trained model makes converged queries take fewer iterations
  than the cold start, with results within 1e-4 of the converged oracle."""
import numpy as np
import pytest

from conftest import rel_err
from oracle import ws_mlp

pytestmark = pytest.mark.gpu


def test_gradient_vs_cpu_oracle(wmd):
    d = 300
    rng = np.random.default_rng(0)
    F, o, n = ws_mlp.layout(d)
    p = wmd.ws_init_params(d, seed=3).astype(np.float64)
    p[o["shift"][0]:o["shift"][0] + F] = rng.normal(size=F) * 0.1
    p[o["scale"][0]:o["scale"][0] + F] = rng.uniform(0.5, 2.0, F)
    for k in ("b1", "b2", "b3"):
        a, m = o[k]
        p[a:a + m] = rng.normal(size=m) * 0.1
    p = p.astype(np.float32)
    X = rng.normal(size=(300, F)).astype(np.float32)
    t = rng.normal(size=300).astype(np.float32)
    gptr = np.array([0, 16, 32, 40, 41, 100, 164, 228, 300], np.int64)
    eng = wmd.Engine()
    loss, g = eng.ws_loss_grad(d, X, t, gptr, p)
    rl, rg = ws_mlp.loss_grad(p.astype(np.float64), d, X.astype(np.float64),
                              t.astype(np.float64), gptr)
    assert abs(loss - rl) <= 1e-4 * abs(rl)
    for k in ("W1", "b1", "W2", "b2", "w3", "b3"):
        a, m = o[k]
        m = 1 if k == "b3" else m
        ref, got = rg[a:a + m], g[a:a + m].astype(np.float64)
        if k == "b3":  # sum of centred errors: exactly 0, FP32 round-off here
            assert abs(got[0]) <= 1e-6
            continue
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-3 * scale, k
    assert np.all(g[:o["W1"][0]] == 0)  # shift/scale are not trained
    eng.close()


@pytest.fixture(scope="module")
def small(synth):
    p = synth.case(3000, 300, 300, 24, 8, 64, 40, 21)
    rs = [synth.source_doc(p.V, v, seed=40 + q) for q, v in enumerate((12, 40, 90))]
    return p, rs


def test_labels_and_features_vs_oracle(wmd, small, oracle_mod):
    p, rs = small
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    info = eng.ws_build_training_set(rs, p.lam, docs_per_source=12, words_per_doc=8,
                                     label_tol=1e-7, label_max_iter=20000, seed=1)
    assert info["groups"] >= 30
    ts = eng.ws_training_set(info)
    params, _ = eng.ws_train(wmd.ws_init_params(300, 0), epochs=1, batch_groups=8)
    F, o, _ = ws_mlp.layout(300)
    shift = params[o["shift"][0]:o["shift"][0] + F]
    scale = params[o["scale"][0]:o["scale"][0] + F]
    Xraw = ts["X"].astype(np.float64) / scale + shift
    for q, r in enumerate(rs):
        ids = np.nonzero(r)[0]
        conv, it, res, U = oracle_mod.sinkhorn_converged(
            r, p.vecs.astype(np.float64), p.col_ptr, p.row_inds, p.vals, p.lam,
            tol=1e-9, max_iter_cap=50000, want_u=True)
        for g in np.nonzero(ts["source"] == q)[0]:
            j = int(ts["doc"][g])
            rows = np.arange(ts["gptr"][g], ts["gptr"][g + 1])
            words = ts["word"][rows]
            np.testing.assert_allclose(ts["y"][rows], np.log(U[j, words]), atol=2e-3)
            ref = ws_mlp.features(p.vecs, p.col_ptr, p.row_inds, p.vals, ids, r[ids],
                                  [(int(i), j) for i in words])
            np.testing.assert_allclose(Xraw[rows, :605], ref[:, :605], rtol=1e-4, atol=2e-4)
    eng.close()


def test_inference_vs_cpu_oracle(wmd, small):
    p, rs = small
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    info = eng.ws_build_training_set(rs, p.lam, docs_per_source=40, words_per_doc=8,
                                     label_tol=1e-6, label_max_iter=20000, seed=2)
    params, loss = eng.ws_train(wmd.ws_init_params(300, 1), epochs=3, batch_groups=16,
                                lr=1e-3)
    assert np.all(np.isfinite(loss))
    eng.set_warm_start(params)
    r = rs[1]
    ids = np.nonzero(r)[0]
    u0 = eng.ws_init_scalings(r, p.lam)
    assert u0.shape == (p.N, ids.size)
    rng = np.random.default_rng(0)
    docs = [j for j in rng.choice(p.N, 40, replace=False) if p.col_ptr[j + 1] > p.col_ptr[j]]
    pairs = [(i, int(j)) for j in docs for i in range(ids.size)]
    X = ws_mlp.features(p.vecs, p.col_ptr, p.row_inds, p.vals, ids, r[ids], pairs)
    y, _ = ws_mlp.forward(params.astype(np.float64), 300, X)
    got = np.log(np.array([u0[j, i] for i, j in pairs], np.float64))
    # u0 is the prediction up to one factor per document (the iteration is
    # invariant to it; the engine sets it so that the largest entry is v_r):
    # compare per-document centred log u, and the largest entry.
    nw = ids.size
    g2, y2 = got.reshape(-1, nw), y.reshape(-1, nw)
    err = np.abs((g2 - g2.mean(1, keepdims=True)) - (y2 - y2.mean(1, keepdims=True)))
    assert err.max() <= 2 * (0.05 + 0.01 * np.abs(y).max()), err.max()
    assert np.allclose(np.exp(g2).max(1), nw, rtol=1e-5)
    eng.close()


def test_end_to_end_gain(wmd, synth, oracle_mod):
    """Trained on 24 sources, evaluated on 3 held-out ones: converged queries
    (marginal residual <= 1e-5) from the warm start take fewer iterations and
    agree with the converged FP64 oracle."""
    p = synth.case(4000, 300, 1500, 24, 8, 96, 40, 31)
    cdf = synth.zipf_cdf(p.V)
    train = [synth.source_doc(p.V, int(v), seed=100 + q, cdf=cdf)
             for q, v in enumerate(np.random.default_rng(5).integers(16, 160, 24))]
    held = [synth.source_doc(p.V, v, seed=900 + v, cdf=cdf) for v in (30, 80, 150)]
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.ws_build_training_set(train, p.lam, docs_per_source=120, words_per_doc=16,
                              label_tol=1e-7, label_max_iter=20000, seed=3)
    params, loss = eng.ws_train(wmd.ws_init_params(300, 2), epochs=8, batch_groups=64,
                                lr=1e-3)
    assert loss[-1] < loss[0]
    eng.set_tolerance(1e-5)
    cold, it_cold = eng.query_batch(held, p.lam, 5000, want_iters=True)
    eng.set_warm_start(params)
    warm, it_warm = eng.query_batch(held, p.lam, 5000, want_iters=True)
    # the warm start combined with over-relaxation of both half-steps
    eng.set_relaxation(1.7)
    warm_rx, it_rx = eng.query_batch(held, p.lam, 5000, want_iters=True)
    eng.set_relaxation(1.0)
    for q, r in enumerate(held):
        conv = oracle_mod.sinkhorn_converged(r, p.vecs.astype(np.float64), p.col_ptr,
                                             p.row_inds, p.vals, p.lam, tol=1e-9,
                                             max_iter_cap=50000)[0]
        done = (it_warm[q] < 5000) & (it_cold[q] < 5000) & (it_rx[q] < 5000)
        assert done.mean() > 0.95
        assert rel_err(warm[q][done], conv[done]).max() <= 1e-4
        assert rel_err(cold[q][done], conv[done]).max() <= 1e-4
        assert rel_err(warm_rx[q][done], conv[done]).max() <= 1e-4
    print(f"mean iterations cold {it_cold.mean():.1f} warm {it_warm.mean():.1f} "
          f"warm + omega 1.7 {it_rx.mean():.1f}")
    assert it_warm.mean() < it_cold.mean()
    assert it_rx.mean() < it_warm.mean()
    eng.close()


def test_gain_on_sources_seen_in_training(wmd, synth, oracle_mod):
    """What a trained network gains when its predictions are good: trained on
    the sources it is then asked about (each source's own converged scalings
    on a sample of the documents), the warm start must cut the mean number of
    updates to a marginal residual of 1e-5 by at least 15 % over the cold
    start (22 % measured on a B200), with the scores within 1e-4 of the
    converged FP64 oracle.  Device time is printed, not asserted: with 1500
    documents per source (about one per resident warp) a query lasts as long
    as its slowest documents, which need thousands of updates from either
    start, so the inference and the second candidate's first update cost more
    than the saved updates (24.3 vs 22.0 ms measured).  On sources it has not
    seen (test_end_to_end_gain, the bench's held-out protocol) the same
    network gains little: its errors lie along the iteration's slow modes."""
    p = synth.case(4000, 300, 1500, 24, 8, 96, 40, 33)
    cdf = synth.zipf_cdf(p.V)
    srcs = [synth.source_doc(p.V, v, seed=700 + v, cdf=cdf) for v in (40, 90, 150)]
    eng = wmd.Engine()
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.ws_build_training_set(srcs, p.lam, docs_per_source=1500, words_per_doc=40,
                              label_tol=1e-7, label_max_iter=20000, seed=4)
    params, loss = eng.ws_train(wmd.ws_init_params(300, 3), epochs=60, batch_groups=64,
                                lr=2e-3)
    eng.set_tolerance(1e-5)
    eng.set_batch_mode(False)
    eng.set_timing(True)
    cold, it_cold = eng.query_batch(srcs, p.lam, 5000, want_iters=True)
    t_cold = sum(eng.stage_times())
    eng.set_warm_start(params)
    warm, it_warm = eng.query_batch(srcs, p.lam, 5000, want_iters=True)
    t_warm = sum(eng.stage_times())
    eng.close()
    for q, r in enumerate(srcs):
        conv = oracle_mod.sinkhorn_converged(r, p.vecs.astype(np.float64), p.col_ptr,
                                             p.row_inds, p.vals, p.lam, tol=1e-9,
                                             max_iter_cap=50000)[0]
        done = (it_warm[q] < 5000) & (it_cold[q] < 5000)
        assert done.mean() > 0.95
        assert rel_err(warm[q][done], conv[done]).max() <= 1e-4
    gain = 1.0 - it_warm.mean() / it_cold.mean()
    print(f"seen sources: updates cold {it_cold.mean():.1f} warm {it_warm.mean():.1f} "
          f"({100 * gain:.0f} % fewer), max cold {it_cold.max()} warm {it_warm.max()}; "
          f"device ms cold {t_cold:.2f} warm {t_warm:.2f}")
    assert gain >= 0.15
