"""fp64 value columns: SUM (and AVG) accumulated in fp64.

The CUDA path adds each fp64 value exactly into the shared table's 128-bit
fixed-point accumulator when its binary expansion lies in [2^-64, 2^30), and
into an fp64 residual otherwise; partial sums meet in HBM through fp64
additions.  The oracle sums each group's rows in fp64 in row order.  Tolerance:
|gpu - oracle| <= 1e-12 * |oracle| + 1e-12 * sum(|x|) over the group (at most a
few hundred fp64 roundings of partial sums no larger than sum(|x|) on either
side).  Integer aggregates beside the fp64 ones stay bit-exact.  Covered: both
strategies, int32 and int64 keys, values outside the exact window (huge, tiny,
negative zero), the batch and host-resident entry points, AVG, and the
refusal of MIN/MAX on fp64 columns."""
import numpy as np
import pytest

import cpu_oracle as O
from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
from gpu_util import run_gpu, sort_result, to_device

pytestmark = pytest.mark.gpu

F64_RTOL = 1e-12
F64_ABS_PER_ABSSUM = 1e-12


def _data(n, kdt, ndv, seed):
    rng = np.random.default_rng(seed)
    dom = rng.integers(np.iinfo(kdt).min, np.iinfo(kdt).max, size=ndv, dtype=np.int64).astype(kdt)
    keys = dom[rng.integers(0, ndv, size=n)]
    f64 = rng.standard_normal(n) * 1e3
    special = rng.random(n)
    f64[special < 0.01] *= 1e12           # |x| >= 2^30: the residual path
    f64[(special >= 0.01) & (special < 0.02)] *= 1e-30   # bits below 2^-64
    f64[(special >= 0.02) & (special < 0.025)] = -0.0
    cols = [f64, rng.integers(-1000, 1000, size=n, dtype=np.int64), rng.standard_normal(n).astype(np.float32)]
    return keys, cols


def _check_fp(got, keys, cols, col, label):
    ok, (s,) = O.groupby(keys, cols, [("sum", col)], nthreads=8)
    _, (a,) = O.groupby(keys, cols, [("sumabs", col)], nthreads=8)
    assert got.dtype == np.float64
    bad = np.abs(got - s) > F64_RTOL * np.abs(s) + F64_ABS_PER_ABSSUM * a
    assert not bad.any(), f"{label}: {bad.sum()} groups off, e.g. {got[bad][:3]} vs {s[bad][:3]}"
    return ok


@pytest.mark.parametrize("strategy", ["table", "partition"])
@pytest.mark.parametrize("kdt", [np.int32, np.int64])
def test_f64_sum_matches_oracle(ctx, strategy, kdt):
    keys, cols = _data(400_009, kdt, 50_000, seed=17)
    aggs = [("sum", 0), ("count", None), ("sum", 1), ("sum", 2)]
    gk, ga, _ = run_gpu(ctx, keys, cols, aggs, knobs=dict(strategy=strategy))
    gk, ga = sort_result(gk, ga, False)
    ok = _check_fp(ga[0], keys, cols, 0, f"{strategy} f64 sum")
    np.testing.assert_array_equal(gk, ok)
    _, (c, s1) = O.groupby(keys, cols, [("count", None), ("sum", 1)], nthreads=8)
    np.testing.assert_array_equal(ga[1], c)
    np.testing.assert_array_equal(ga[2], s1)
    _check_fp(ga[3], keys, cols, 2, f"{strategy} f32 sum beside f64")


def test_f64_few_hot_keys(ctx):
    """Eight keys over a million rows: every CTA's shared table holds every key."""
    keys, cols = _data(1 << 20, np.int64, 8, seed=5)
    gk, ga, _ = run_gpu(ctx, keys, cols, [("sum", 0)])
    gk, ga = sort_result(gk, ga, False)
    np.testing.assert_array_equal(gk, _check_fp(ga[0], keys, cols, 0, "hot keys"))


def test_f64_avg_and_sorted(ctx):
    keys, cols = _data(100_000, np.int32, 3_000, seed=9)
    gk, ga, _ = run_gpu(ctx, keys, cols, [("avg", 0), ("count", None)], knobs=dict(sort_output=1))
    ok, (s, c) = O.groupby(keys, cols, [("sum", 0), ("count", None)], nthreads=8)
    _, (a,) = O.groupby(keys, cols, [("sumabs", 0)], nthreads=8)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(ga[1], c)
    avg = s / c
    assert (np.abs(ga[0] - avg) <= F64_RTOL * np.abs(avg) + F64_ABS_PER_ABSSUM * a / c).all()


def test_f64_batch_and_host(ctx):
    host = [_data(n, kdt, ndv, seed=sd) for n, kdt, ndv, sd in
            [(60_000, np.int64, 500, 1), (90_000, np.int32, 40_000, 2), (2_000, np.int64, 2_000, 3)]]
    aggs = [("sum", 0), ("max", 1)]
    qs = [(to_device(k), [to_device(c) for c in cols], aggs) for k, cols in host]
    res = ctx.groupby_batch(qs)
    for qi, ((keys, cols), r) in enumerate(zip(host, res)):
        gk, ga = sort_result(r.keys.cpu().numpy(), [t.cpu().numpy() for t in r.aggs], False)
        np.testing.assert_array_equal(gk, _check_fp(ga[0], keys, cols, 0, f"batch query {qi}"))
        np.testing.assert_array_equal(ga[1], O.groupby(keys, cols, [("max", 1)], nthreads=8)[1][0])
    keys, cols = host[1]
    r = ctx.groupby_host(keys, cols, aggs)
    gk, ga = sort_result(np.asarray(r.keys), [np.asarray(a) for a in r.aggs], False)
    np.testing.assert_array_equal(gk, _check_fp(ga[0], keys, cols, 0, "host-resident"))


@pytest.mark.parametrize("op", ["min", "max"])
def test_f64_min_max_refused(ctx, op):
    keys, cols = _data(1000, np.int64, 10, seed=1)
    with pytest.raises(A.GbaError) as e:
        run_gpu(ctx, keys, cols, [(op, 0)])
    assert e.value.status == A.ERR_UNSUPPORTED
