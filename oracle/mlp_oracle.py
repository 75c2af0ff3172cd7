"""TEST INFRASTRUCTURE ONLY -- CPU oracle of the cost-model MLP.

Float64 numpy restatement of the network in mex_linear_algebra_b200/csrc/
mlp.cu (10 -> 32 ReLU -> 32 ReLU -> 10, flat parameters W1 b1 W2 b2 W3 b3,
masked mean squared error), with analytic gradients.  The GPU kernels are
checked against it, and it is checked against central finite differences.
The reference library has no learned component; this oracle pins the
project's own kernels.
"""
import numpy as np

IN, H1, H2, OUT = 10, 32, 32, 10
SHAPES = [("W1", (IN, H1)), ("b1", (H1,)), ("W2", (H1, H2)), ("b2", (H2,)), ("W3", (H2, OUT)),
          ("b3", (OUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(p):
    out, o = {}, 0
    for name, shp in SHAPES:
        k = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + k], dtype=np.float64).reshape(shp)
        o += k
    return out


def flatten(d):
    return np.concatenate([d[name].ravel() for name, _ in SHAPES])


def init(seed=0):
    rng = np.random.default_rng(seed)
    d = {}
    for name, shp in SHAPES:
        if name.startswith("W"):
            d[name] = rng.normal(0, np.sqrt(2.0 / shp[0]), size=shp)
        else:
            d[name] = np.zeros(shp)
    return flatten(d)


def forward(p, X):
    P = unflatten(p)
    X = np.asarray(X, dtype=np.float64)
    a1 = X @ P["W1"] + P["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ P["W2"] + P["b2"]
    h2 = np.maximum(a2, 0)
    y = h2 @ P["W3"] + P["b3"]
    return y, (X, a1, h1, a2, h2)


def loss_and_grad(p, X, T, M):
    """Masked MSE: sum(M*(y-T)^2) / sum(M); analytic gradient (flat)."""
    P = unflatten(p)
    y, (X, a1, h1, a2, h2) = forward(p, X)
    cnt = max(float(np.sum(M != 0)), 1.0)
    e = np.where(M != 0, y - T, 0.0)
    loss = float(np.sum(e * e)) / cnt
    dy = 2.0 * e / cnt
    g = {"W3": h2.T @ dy, "b3": dy.sum(0)}
    dh2 = (dy @ P["W3"].T) * (a2 > 0)
    g["W2"] = h1.T @ dh2
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ P["W2"].T) * (a1 > 0)
    g["W1"] = X.T @ dh1
    g["b1"] = dh1.sum(0)
    return loss, flatten(g)


def numeric_grad(p, X, T, M, eps=1e-6):
    g = np.zeros_like(p, dtype=np.float64)
    for i in range(len(p)):
        q = p.astype(np.float64).copy()
        q[i] += eps
        lp, _ = loss_and_grad(q, X, T, M)
        q[i] -= 2 * eps
        lm, _ = loss_and_grad(q, X, T, M)
        g[i] = (lp - lm) / (2 * eps)
    return g
