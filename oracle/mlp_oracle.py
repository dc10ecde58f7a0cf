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


# ---------------------------------------------------------------------------
# Estimator features: a numpy restatement of the sampling and reduction
# kernels (csrc/k_est.cu: sample_row, k_est_sample, k_est_reduce), for
# checking them.  Defaults follow csrc/est_kernels.h (at most 256 sampled
# tiles of 65536 rows, 1024 sampled rows per tile).
EST_MAX_TILES = 256
EST_SEED = 0x5BD1E995


def _rotl32(x: np.ndarray, r: int) -> np.ndarray:
    return (x << np.uint32(r)) | (x >> np.uint32(32 - r))


def _mm3_round(h: np.ndarray, k: np.ndarray) -> np.ndarray:
    k = k * np.uint32(0xCC9E2D51)
    k = _rotl32(k, 15)
    k = k * np.uint32(0x1B873593)
    h = h ^ k
    h = _rotl32(h, 13)
    return h * np.uint32(5) + np.uint32(0xE6546B64)


def _mm3_fmix(h: np.ndarray) -> np.ndarray:
    h = h ^ (h >> np.uint32(16))
    h = h * np.uint32(0x85EBCA6B)
    h = h ^ (h >> np.uint32(13))
    h = h * np.uint32(0xC2B2AE35)
    return h ^ (h >> np.uint32(16))


def murmur3_keys(keys: np.ndarray, key64: bool, seed: int = EST_SEED) -> np.ndarray:
    """MurmurHash3 (x86, 32-bit) of every key's 4 or 8 little-endian bytes."""
    with np.errstate(over="ignore"):
        h = np.full(keys.shape[0], seed, dtype=np.uint32)
        if key64:
            k = keys.astype(np.uint64)
            h = _mm3_round(h, (k & np.uint64(0xFFFFFFFF)).astype(np.uint32))
            h = _mm3_round(h, (k >> np.uint64(32)).astype(np.uint32))
            return _mm3_fmix(h ^ np.uint32(8))
        h = _mm3_round(h, keys.astype(np.uint32))
        return _mm3_fmix(h ^ np.uint32(4))


def sampled_rows(n: int, tile_rows: int = 65536) -> np.ndarray:
    """Row indices the sampling kernel reads (sample_row over every item)."""
    ntiles = (n + tile_rows - 1) // tile_rows
    step = max(1, (ntiles + EST_MAX_TILES - 1) // EST_MAX_TILES)
    out = []
    for t in range(0, ntiles, step):
        tb = t * tile_rows
        ln = min(tb + tile_rows, n) - tb
        if ln <= 1024:
            out.append(np.arange(tb, tb + ln, dtype=np.int64))
        else:
            j = np.arange(1024, dtype=np.int64)
            out.append(tb + (j >> 3) * (ln // 128) + (j & 7))
    return np.concatenate(out) if out else np.zeros(0, dtype=np.int64)


def est_features(keys: np.ndarray, key64: bool, tile_rows: int = 65536) -> np.ndarray:
    """The 32 features of a key column, as k_est_reduce computes them."""
    n = int(keys.shape[0])
    rows = sampled_rows(n, tile_rows)
    k = keys.view(np.uint64 if key64 else np.uint32)[rows] if n else np.zeros(0, np.uint32)
    h = murmur3_keys(k, key64)
    reg = (h >> np.uint32(26)).astype(np.int64)
    x = ((h << np.uint32(6)) | np.uint32(32)).astype(np.uint64)
    rank = 32 - np.floor(np.log2(x.astype(np.float64))).astype(np.int64)  # clz(x) + 1
    hll = np.zeros(64, dtype=np.int64)
    np.maximum.at(hll, reg, rank)
    _, cnt = np.unique(k, return_counts=True)
    s = float(max(len(rows), 1))
    dd = float(len(cnt))
    a = [float(np.sum(cnt == c)) for c in (1, 2, 3)] + [float(np.sum(cnt >= 4))]
    mx = float(cnt.max()) if len(cnt) else 0.0
    nf = float(n)
    gee = np.sqrt(nf / s) * a[0] + (dd - a[0])
    chao = dd + a[0] * a[0] / (2.0 * (a[1] if a[1] > 1 else 1.0))
    z = float(np.sum(np.ldexp(1.0, -hll)))
    zeros = int(np.sum(hll == 0))
    est = 0.709 * 64 * 64 / z
    if est <= 2.5 * 64 and zeros > 0:
        est = 64 * np.log(64.0 / zeros)
    f = np.zeros(F, dtype=np.float64)
    f[0] = np.log2(nf + 1) / 32
    f[1] = np.log2(s + 1) / 32
    f[2], f[3], f[4], f[5], f[6] = dd / s, a[0] / s, a[1] / s, a[2] / s, a[3] / s
    f[7] = np.log2(dd + 1) / 32
    f[8] = np.log2(gee + 1) / 32
    f[9] = np.log2(chao + 1) / 32
    f[10] = np.log2(est + 1) / 32
    f[11] = mx / s
    f[12] = 1.0 if key64 else 0.5
    f[13] = s / (nf if nf > 0 else 1)
    f[14:30] = np.bincount(np.minimum(hll, 15), minlength=16) / 64.0
    f[30] = np.log2(max(nf / s, 1.0)) / 32
    f[31] = 1.0
    return f.astype(np.float32)
