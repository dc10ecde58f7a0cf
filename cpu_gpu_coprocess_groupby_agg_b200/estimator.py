"""Learned cardinality estimator: weights, training set, training, evaluation.

The network (32 features -> 3 x 64 ReLU -> log2(groups)/32) lives in
libgba.so: features, forward, backward and Adam are CUDA kernels there
(csrc/k_est.cu).  This module draws the training tables, labels them with the
exact group count the plain method returns, trains on the GPU and stores the
weights next to this file (estimator_weights.f32).
"""
from __future__ import annotations

import math
import time
from pathlib import Path

import numpy as np

from . import _abi as A

WEIGHTS = Path(__file__).resolve().parent / "estimator_weights.f32"
F, H = A.GBA_EST_FEATURES, A.GBA_EST_HIDDEN
# parameter layout (matches csrc/k_est.cu)
SHAPES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
          ("W4", (H,)), ("b4", (1,))]


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases, output bias 0.5 (t ~ log2(G)/32)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        if name.startswith("W"):
            fan_in = shape[-1] if len(shape) == 2 else shape[0]
            lim = math.sqrt(6.0 / fan_in) * (0.5 if name == "W4" else 1.0)
            parts.append(rng.uniform(-lim, lim, size=shape).astype(np.float32).ravel())
        elif name == "b4":
            parts.append(np.array([0.5], dtype=np.float32))
        else:
            parts.append(np.zeros(shape, dtype=np.float32).ravel())
    return np.concatenate(parts)


def load_weights() -> np.ndarray:
    """The committed estimator weights (fp32, gba_estimator_param_count values)."""
    return np.fromfile(WEIGHTS, dtype=np.float32)


def load_default(ctx) -> bool:
    """Loads the committed weights into ctx; False when the file is absent."""
    if not WEIGHTS.exists():
        return False
    ctx.est_load(np.fromfile(WEIGHTS, dtype=np.float32))
    return True


def draw_shape(rng: np.random.Generator, min_log2: float = 12.0, max_log2: float = 24.0):
    """One table shape from the batch-workload distribution."""
    n = int(round(2 ** rng.uniform(min_log2, max_log2)))
    ndv = int(round(math.exp(rng.uniform(math.log(16), math.log(max(17, n // 2))))))
    s = float(rng.uniform(0.0, 1.5))
    bits = 64 if rng.random() < 0.5 else 32
    return n, ndv, s, bits


def make_training_set(ctx, count: int, seed: int = 1234, min_log2: float = 12.0, max_log2: float = 24.0,
                      device: int = 0, log_every: int = 0):
    """(features [count, 32], log2 exact groups [count], shapes) on the GPU.

    Each table is generated on the device, its features computed by the
    library's sampling kernels, and its exact group count taken from a plain
    (estimator-free) GROUP BY COUNT of the same column.
    """
    import torch
    from .api import gen_device, gen_spec
    rng = np.random.default_rng(seed)
    X = np.empty((count, F), dtype=np.float32)
    y = np.empty(count, dtype=np.float32)
    shapes = []
    t0 = time.time()
    for i in range(count):
        n, ndv, s, bits = draw_shape(rng, min_log2, max_log2)
        sp = gen_spec(seed * 7919 + i, bits, ndv, s, [])
        keys, _ = gen_device(sp, n, device=device)
        X[i] = ctx.est_features(keys)
        res = ctx.groupby(keys, [], [("count", None)], knobs={"sizing": "plain"}, capacity=min(n, 2 * ndv) + 2)
        y[i] = math.log2(max(res.n_groups, 1))
        shapes.append((n, ndv, s, bits))
        del keys
        if log_every and (i + 1) % log_every == 0:
            print(f"  {i + 1}/{count} tables, {time.time() - t0:.1f}s", flush=True)
    torch.cuda.synchronize()
    return X, y, shapes


def q_error(pred_log2: np.ndarray, true_log2: np.ndarray) -> np.ndarray:
    return np.exp2(np.abs(pred_log2 - true_log2))


def classical_estimates(X: np.ndarray) -> dict:
    """log2 estimates of the classical sample estimators carried in the features."""
    return {"gee": X[:, 8] * 32, "chao1": X[:, 9] * 32, "sample_distinct": X[:, 7] * 32,
            "plain_rows": X[:, 0] * 32}


def train(ctx, X: np.ndarray, y: np.ndarray, epochs: int = 150, batch: int = 128, lr: float = 2e-3,
          seed: int = 0) -> float:
    ctx.est_load(init_params(seed))
    return ctx.est_train(X, y, epochs=epochs, batch=batch, lr=lr, seed=seed)


def evaluate(ctx, X: np.ndarray, y: np.ndarray) -> dict:
    pred = ctx.est_predict(X)
    # the library clamps to [sample distinct, rows]; do the same here
    lo, hi = X[:, 7] * 32, X[:, 0] * 32
    pred = np.clip(pred, np.log2(np.maximum(np.exp2(lo) - 1, 1)), hi)
    out = {"learned": q_error(pred, y)}
    for k, v in classical_estimates(X).items():
        out[k] = q_error(v, y)
    return {k: {"median": float(np.median(v)), "p90": float(np.percentile(v, 90)),
                "p99": float(np.percentile(v, 99)), "max": float(v.max())} for k, v in out.items()}
