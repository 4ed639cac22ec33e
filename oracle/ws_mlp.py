"""CPU oracle (float64) of the learned warm start's network -- test
infrastructure only (tests and the bench's checks import it; the library
never does).

The reference has no warm start (it always starts from u = v_r,
sinkhorn_wmd_fused.cpp:188-191); this module restates the network the GPU
kernels implement so that their forward pass, loss and gradients can be
checked:

    x~  = (x - shift) * scale                       (per feature)
    h1  = gelu(W1 x~ + b1)      W1 [256][F]
    h2  = gelu(W2 h1 + b2)      W2 [256][256]
    y   = w3 . h2 + b3          (prediction of log u_i)
    loss = sum_g sum_{m in g} (e_m - mean_g e)^2 / P,  e = y - t

with the tanh form of GELU.  Parameter vector layout (float32 on the GPU):
shift[F], scale[F], W1, b1, W2, b2, w3, b3 (+3 pad), F = 2d + 5 rounded up
to 16.  Feature row of (source word i, document j): embedding of i [d],
c-weighted centroid of j [d], r_i, log r_i, min / mean / max over j's words
w of M(i, w) = |E_i - E_w|, zero padding.
"""
import numpy as np

H = 256
C0 = np.sqrt(2.0 / np.pi)


def layout(d):
    F = ((2 * d + 5) + 15) // 16 * 16
    o = {}
    pos = 0
    for name, n in (("shift", F), ("scale", F), ("W1", H * F), ("b1", H),
                    ("W2", H * H), ("b2", H), ("w3", H), ("b3", 4)):
        o[name] = (pos, n)
        pos += n
    return F, o, pos


def unpack(params, d):
    F, o, n = layout(d)
    p = np.asarray(params, np.float64)
    assert p.size == n
    g = {k: p[a:a + m] for k, (a, m) in o.items()}
    g["W1"] = g["W1"].reshape(H, F)
    g["W2"] = g["W2"].reshape(H, H)
    g["b3"] = g["b3"][:1]
    return g


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(C0 * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(C0 * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C0 * (1.0 + 3 * 0.044715 * z * z)


def forward(params, d, X):
    g = unpack(params, d)
    Xs = (np.asarray(X, np.float64) - g["shift"]) * g["scale"]
    Z1 = Xs @ g["W1"].T + g["b1"]
    H1 = gelu(Z1)
    Z2 = H1 @ g["W2"].T + g["b2"]
    H2 = gelu(Z2)
    y = H2 @ g["w3"] + g["b3"][0]
    return y, (Xs, Z1, H1, Z2, H2)


def loss_grad(params, d, X, t, gptr):
    """Loss and gradient (same layout as params; zero for shift/scale)."""
    F, o, n = layout(d)
    g = unpack(params, d)
    y, (Xs, Z1, H1, Z2, H2) = forward(params, d, X)
    P = y.size
    e = y - np.asarray(t, np.float64)
    dy = np.empty(P)
    loss = 0.0
    for a, b in zip(gptr[:-1], gptr[1:]):
        ec = e[a:b] - e[a:b].mean()
        loss += (ec ** 2).sum() / P
        dy[a:b] = 2.0 * ec / P
    grad = np.zeros(n)
    put = lambda k, v: grad.__setitem__(slice(o[k][0], o[k][0] + v.size), v.ravel())
    put("w3", H2.T @ dy)
    put("b3", np.array([dy.sum()]))
    dZ2 = np.outer(dy, g["w3"]) * gelu_grad(Z2)
    put("b2", dZ2.sum(0))
    put("W2", dZ2.T @ H1)
    dZ1 = (dZ2 @ g["W2"]) * gelu_grad(Z1)
    put("b1", dZ1.sum(0))
    put("W1", dZ1.T @ Xs)
    return loss, grad


def features(E, col_ptr, row_inds, vals, src_ids, src_w, pairs):
    """Raw feature rows for (source word index i, document j) pairs, M exact
    in float64 from the embeddings."""
    E = np.asarray(E, np.float64)
    d = E.shape[1]
    F = layout(d)[0]
    X = np.zeros((len(pairs), F))
    for m, (i, j) in enumerate(pairs):
        a, b = col_ptr[j], col_ptr[j + 1]
        w, c = row_inds[a:b], vals[a:b]
        wi = src_ids[i]
        X[m, :d] = E[wi]
        X[m, d:2 * d] = (c[:, None] * E[w]).sum(0) / c.sum()
        X[m, 2 * d] = src_w[i]
        X[m, 2 * d + 1] = np.log(src_w[i])
        M = np.sqrt(((E[w] - E[wi]) ** 2).sum(1))
        X[m, 2 * d + 2:2 * d + 5] = (M.min(), M.mean(), M.max())
    return X
