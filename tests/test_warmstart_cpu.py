"""CPU: the warm-start network's CPU oracle (finite differences pin its
gradient) and the host-side parameter initialisation."""
import numpy as np

from oracle import ws_mlp


def _problem(d=3, P=40, seed=0):
    rng = np.random.default_rng(seed)
    F, o, n = ws_mlp.layout(d)
    p = np.zeros(n)
    p[o["shift"][0]:o["shift"][0] + F] = rng.normal(size=F) * 0.1
    p[o["scale"][0]:o["scale"][0] + F] = rng.uniform(0.5, 2.0, F)
    for k in ("W1", "b1", "W2", "b2", "w3", "b3"):
        a, m = o[k]
        p[a:a + m] = rng.normal(size=m) * 0.2
    X = rng.normal(size=(P, F))
    t = rng.normal(size=P)
    gptr = np.array([0, 5, 12, 13, 25, 40])
    return p, X, t, gptr, o


def test_oracle_gradient_matches_finite_differences():
    d = 3
    p, X, t, gptr, o = _problem(d)
    loss, g = ws_mlp.loss_grad(p, d, X, t, gptr)
    rng = np.random.default_rng(1)
    for k in ("W1", "b1", "W2", "b2", "w3", "b3"):
        a, m = o[k]
        m = 1 if k == "b3" else m
        for idx in rng.choice(m, size=min(m, 6), replace=False):
            e = np.zeros_like(p)
            e[a + idx] = 1e-6
            fd = (ws_mlp.loss_grad(p + e, d, X, t, gptr)[0] -
                  ws_mlp.loss_grad(p - e, d, X, t, gptr)[0]) / 2e-6
            assert abs(fd - g[a + idx]) <= 1e-6 + 1e-5 * abs(fd), (k, idx, fd, g[a + idx])
    # the centred loss ignores a per-group offset of the targets
    t2 = t.copy()
    t2[5:12] += 3.0
    assert np.isclose(ws_mlp.loss_grad(p, d, X, t2, gptr)[0], loss)


def test_param_layout_and_init(wmd):
    for d in (3, 300):
        n = wmd.ws_param_count(d)
        F, o, n2 = ws_mlp.layout(d)
        assert n == n2
        p = wmd.ws_init_params(d, seed=5)
        assert p.shape == (n,) and p.dtype == np.float32
        assert np.all(p[o["shift"][0]:o["shift"][0] + F] == 0)
        assert np.all(p[o["scale"][0]:o["scale"][0] + F] == 1)
        W1 = p[o["W1"][0]:o["W1"][0] + o["W1"][1]]
        assert abs(W1.std() * np.sqrt(F) - 1.0) < 0.05
        np.testing.assert_array_equal(p, wmd.ws_init_params(d, seed=5))
