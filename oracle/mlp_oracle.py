"""Float64 numpy restatement of the estimator MLP (forward, MSE loss, backward).

TEST INFRASTRUCTURE ONLY: the checker for the GPU gradient kernels
(csrc/k_est.cu k_mlp_fwd_bwd).  Layout and semantics follow that kernel:
32 inputs -> 64 -> 64 -> 64 (ReLU) -> 1, target t = log2(groups)/32,
loss = mean((y - t)^2).  The reference repository has no estimator; there is
nothing of it to restate.
"""
import numpy as np

F, H = 32, 64


def unpack(p: np.ndarray) -> dict:
    p = p.astype(np.float64)
    o = 0
    out = {}
    for name, shape in [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
                        ("b3", (H,)), ("W4", (H,)), ("b4", (1,))]:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def forward_backward(p: np.ndarray, X: np.ndarray, log2_groups: np.ndarray):
    """(loss, flat gradient) in float64."""
    w = unpack(p)
    x = X.astype(np.float64)
    t = log2_groups.astype(np.float64) / 32.0
    B = x.shape[0]
    z1 = x @ w["W1"].T + w["b1"]
    a1 = np.maximum(z1, 0)
    z2 = a1 @ w["W2"].T + w["b2"]
    a2 = np.maximum(z2, 0)
    z3 = a2 @ w["W3"].T + w["b3"]
    a3 = np.maximum(z3, 0)
    y = a3 @ w["W4"] + w["b4"][0]
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2 * e / B
    g = {}
    g["W4"] = dy @ a3
    g["b4"] = np.array([dy.sum()])
    d3 = np.outer(dy, w["W4"]) * (z3 > 0)
    g["W3"] = d3.T @ a2
    g["b3"] = d3.sum(0)
    d2 = (d3 @ w["W3"]) * (z2 > 0)
    g["W2"] = d2.T @ a1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ w["W2"]) * (z1 > 0)
    g["W1"] = d1.T @ x
    g["b1"] = d1.sum(0)
    flat = np.concatenate([g[k].ravel() for k in ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"]])
    return loss, flat, y * 32.0
