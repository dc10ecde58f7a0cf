"""Learned cardinality estimator: the GPU kernels against a float64 numpy
oracle, training, and what the trained network gains over plain sizing."""
import math

import numpy as np
import pytest

import mlp_oracle as M
from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E


def test_oracle_gradient_matches_finite_differences():
    """Pins the numpy oracle itself (CPU)."""
    rng = np.random.default_rng(0)
    p = E.init_params(3).astype(np.float64)
    X = rng.random((7, M.F))
    y = rng.uniform(2, 20, size=7)
    loss, g, _ = M.forward_backward(p, X, y)
    for i in rng.choice(len(p), size=40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.forward_backward(pp, X, y)[0] - M.forward_backward(pm, X, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_param_layout_size():
    assert sum(int(np.prod(s)) for _, s in E.SHAPES) == len(E.init_params())


@pytest.mark.gpu
def test_gpu_gradient_matches_oracle(ctx):
    rng = np.random.default_rng(1)
    p = E.init_params(5)
    ctx.est_load(p)
    X = rng.random((96, M.F)).astype(np.float32)
    y = rng.uniform(3, 25, size=96).astype(np.float32)
    g, loss = ctx.est_grad(X, y)
    ref_loss, ref_g, _ = M.forward_backward(p, X, y)
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss) + 1e-7
    scale = np.abs(ref_g).max()
    np.testing.assert_allclose(g, ref_g, rtol=1e-3, atol=1e-4 * scale)


@pytest.mark.gpu
def test_gpu_forward_matches_oracle(ctx):
    rng = np.random.default_rng(2)
    p = E.init_params(7)
    ctx.est_load(p)
    X = rng.random((300, M.F)).astype(np.float32)
    pred = ctx.est_predict(X)
    _, _, ref = M.forward_backward(p, X, np.zeros(300))
    np.testing.assert_allclose(pred, ref, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_features_on_known_columns(ctx):
    import torch
    # 100k rows over exactly 1000 ids: the sample sees all of them
    keys = torch.arange(100_000, dtype=torch.int64, device="cuda") % 1000
    f = ctx.est_features(keys)
    assert abs(f[0] * 32 - math.log2(100_001)) < 1e-3
    assert abs(f[7] * 32 - math.log2(1001)) < 1e-3   # distinct in sample
    assert f[12] == 1.0 and f[31] == 1.0
    assert abs(f[14:30].sum() - 1.0) < 1e-5          # register histogram sums to 1


def test_feature_oracle_hash_matches_murmur3():
    """The numpy feature oracle's MurmurHash3 against the C oracle's (which the
    known-answer vectors pin), on 32- and 64-bit keys (CPU)."""
    import cpu_oracle as O
    rng = np.random.default_rng(3)
    for key64 in (False, True):
        ks = rng.integers(0, 2**63 if key64 else 2**32, size=300, dtype=np.uint64)
        ks = ks if key64 else ks.astype(np.uint32)
        h = M.murmur3_keys(ks, key64)
        assert all(int(h[i]) == O.murmur3_32(ks[i].tobytes(), M.EST_SEED) for i in range(len(ks)))


def test_feature_oracle_sample_layout():
    """Sampled rows: 1024 per sampled tile (128 runs of 8), every row of a
    tile of at most 1024 rows, every step-th tile past 256 tiles (CPU)."""
    r = M.sampled_rows(65536 * 3 + 700)
    assert len(r) == 3 * 1024 + 700 and r.max() == 65536 * 3 + 699
    assert np.array_equal(r[:8], np.arange(8)) and r[8] == 512
    r = M.sampled_rows(65536 * 300)
    assert len(r) == 150 * 1024 and r[1024] == 2 * 65536


def _feature_columns():
    """(name, device key tensor): uniform, skewed, 32- and 64-bit, ragged last
    tile, a single short tile, strided tiles, negative keys, the all-ones key."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(11)
    out = [("1000 ids", torch.arange(100_000, dtype=torch.int64, device="cuda") % 1000),
           ("500 rows", torch.randint(0, 50, (500,), dtype=torch.int32, device="cuda", generator=g)),
           ("ragged i32", torch.randint(-5000, 5000, (65536 * 3 + 700,), dtype=torch.int32, device="cuda",
                                        generator=g))]
    u = torch.rand(3_000_000, device="cuda", generator=g, dtype=torch.float64)
    out.append(("skewed i32", (1.0 / (u + 1e-4)).to(torch.int32)))          # a heavy head and a long tail
    out.append(("strided i64", torch.randint(-2**62, 2**62, (20_000_003,), dtype=torch.int64, device="cuda",
                                             generator=g)))
    ones = torch.randint(0, 300, (1_000_000,), dtype=torch.int64, device="cuda", generator=g)
    ones[::3] = -1                                                             # all-ones key, a third of the rows
    out.append(("all-ones i64", ones))
    return out


@pytest.mark.gpu
def test_features_match_oracle(ctx):
    """All 32 features of the sampling and reduction kernels against the numpy
    restatement of both (same sampled rows, hashes, counts and formulas)."""
    for name, keys in _feature_columns():
        f = ctx.est_features(keys)
        ref = M.est_features(keys.cpu().numpy(), keys.dtype == __import__("torch").int64)
        np.testing.assert_allclose(f, ref, rtol=1e-6, atol=1e-7, err_msg=name)


@pytest.mark.gpu
def test_training_learns_and_beats_plain(ctx):
    """A small training run: loss falls, and the learned estimate's q-error is
    far below plain sizing's (which can only assume groups = rows)."""
    X, y, shapes = E.make_training_set(ctx, 600, seed=7, min_log2=10, max_log2=16)
    ctx.est_load(E.init_params(1))
    p0 = ctx.est_predict(X[:500])
    loss0 = float(np.mean((p0 - y[:500]) ** 2))
    loss = ctx.est_train(X[:500], y[:500], epochs=120, batch=64, lr=3e-3, seed=1)
    assert loss < 0.5 * loss0
    ev = E.evaluate(ctx, X[500:], y[500:])
    assert ev["learned"]["median"] < 1.6
    assert ev["learned"]["median"] < ev["plain_rows"]["median"]


@pytest.mark.gpu
def test_learned_sizing_results_exact(ctx):
    """Results never depend on the estimate: under- and over-estimates only
    change the table size (regrow / larger table)."""
    from gpu_util import compare, run_gpu
    from test_gpu_parity import AGGS_ALL, _data
    if not E.load_default(ctx):
        ctx.est_load(E.init_params(0))
    for n, ndv, z in [(300_000, 50, 0.0), (500_000, 200_000, 0.0), (400_000, 60_000, 1.1)]:
        keys, cols = _data(n, np.int64, ndv, seed=n, zipf=z)
        gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=dict(sizing="learned", learned_min_rows=-1))
        assert res.stats["predicted_groups"] > 0
        compare(gk, ga, keys, cols, AGGS_ALL, f"learned n={n} ndv={ndv}")
    # a deliberately useless network (predicts 1 group) still gives exact results
    bad = E.init_params(0)
    bad[:] = 0
    ctx.est_load(bad)
    keys, cols = _data(200_000, np.int64, 150_000, seed=3)
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=dict(sizing="learned", strategy="table",
                                                                learned_min_rows=-1))
    assert res.stats["predicted_groups"] > 0
    compare(gk, ga, keys, cols, AGGS_ALL, "learned with a useless network")
    # a small query under learned sizing is sized plainly unless told otherwise
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=dict(sizing="learned"))
    assert res.stats["predicted_groups"] < 0
    compare(gk, ga, keys, cols, AGGS_ALL, "learned sizing of a small query")
