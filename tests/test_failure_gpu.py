"""GPU: failure paths, exercised without faulting or hanging the GPU.

* Bounded device waits: a wait that nothing completes gives up after its
  limit, the handle reports WMD_ERR_DEVICE_TIMEOUT at the next check, and the
  same handle then solves correctly (the CUDA context stays usable).
* Warm-start fallback: the solve evaluates the first update from both the
  model's scalings and the cold start and keeps the model's only when its
  marginal residual is not worse (no reference counterpart: the reference
  always starts from u = v_r, sinkhorn_wmd_fused.cpp:188-191).  A model that
  predicts non-finite or wildly wrong scalings must therefore give exactly the
  cold-start results and iteration counts.
"""
import numpy as np
import pytest

from conftest import rel_err
from oracle import ws_mlp

pytestmark = pytest.mark.gpu

WMD_ERR_DEVICE_TIMEOUT = 7


def test_bounded_wait_gives_up_and_handle_recovers(wmd, synth, oracle_mod):
    import time
    p = synth.case(2000, 300, 64, 32, 8, 128, 50, 30)
    eng = wmd.Engine(0)
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    t0 = time.perf_counter()
    st = eng.selftest_bounded_wait(20_000_000)  # 20 ms limit
    dt = time.perf_counter() - t0
    assert st == WMD_ERR_DEVICE_TIMEOUT
    assert b"timed out" in wmd.lib().wmd_last_error()
    assert dt < 1.5, f"the bounded wait took {dt:.2f} s to give up"
    # the error word was cleared and the context still works
    eng.check()
    got = eng.query(p.r, p.lam, p.max_iter)
    ref = oracle_mod.sinkhorn(p.r, p.vecs.astype(np.float64), p.col_ptr,
                              p.row_inds, p.vals, p.lam, p.max_iter)
    assert rel_err(got, ref).max() <= 1e-5
    with pytest.raises(wmd.WMDError):
        eng.selftest_bounded_wait(10)  # limit below 1 us is refused
    eng.close()


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
@pytest.mark.parametrize("kind", ["constant", "wild"])
def test_warm_start_fallback_to_cold_start(wmd, synth, prec, kind):
    """'wild': finite, wildly varying predictions; every document must fall
    back, giving the cold start's results and counts bit for bit.
    'constant': a huge constant prediction (every log u at its clamp): the
    same point as the cold start up to the scale the iteration ignores, so
    the results must agree with the cold start's within the stopping
    tolerance, in about as many updates."""
    p = synth.case(3000, 300, 200, 24, 8, 96, 40, 31)
    held = [synth.source_doc(p.V, v, seed=700 + v) for v in (20, 48, 120)]
    F, o, _ = ws_mlp.layout(300)
    params = wmd.ws_init_params(300, 5).copy()
    a3, _ = o["b3"]
    aw, mw = o["w3"]
    if kind == "constant":
        params[a3] = 1.0e4  # log u clamped to its upper bound for every pair
    else:
        # finite but wildly varying log u per (word, document)
        rng = np.random.default_rng(9)
        params[aw:aw + mw] = rng.normal(size=mw).astype(np.float32) * 20.0
    eng = wmd.Engine(0)
    eng.set_embeddings(p.vecs)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.set_solve_precision(prec)
    eng.set_tolerance(1e-5)
    cold, it_cold = eng.query_batch(held, p.lam, 3000, want_iters=True)
    eng.set_warm_start(params)
    u0 = eng.ws_init_scalings(held[1], p.lam)
    if kind == "wild":
        assert np.isfinite(u0).mean() > 0.5  # the prediction itself is finite
    warm, it_warm = eng.query_batch(held, p.lam, 3000, want_iters=True)
    eng.close()
    if kind == "wild":
        assert np.array_equal(it_warm, it_cold)
        same = (warm == cold) | (np.isnan(warm) & np.isnan(cold))
        assert same.all(), f"{(~same).sum()} documents differ from the cold start"
    else:
        done = (it_warm < 3000) & (it_cold < 3000)
        assert done.mean() > 0.98
        assert abs(it_warm.mean() - it_cold.mean()) <= 0.02 * it_cold.mean()
        assert rel_err(warm[done], cold[done]).max() <= 1e-4
