"""AVG through gba_groupby: the double SUM / COUNT of each group.

Integer columns: the oracle's exact int64 sum rounded to double and divided by
the count is the same IEEE computation the kernel does, so the result is
bit-exact.  fp32 columns: the sums are fp64 in different orders, so the
averages agree to the fp32-SUM tolerance (1e-6 relative, plus the FP64
oracle's own rounding bound for nearly cancelling sums; tests/gpu_util.py).  AVG is checked with and without a COUNT of its own in
the query, on the table and the partition strategy, with learned sizing, and through the
batch entry point."""
import numpy as np
import pytest

import cpu_oracle as O
from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E
from gpu_util import fp_bound, run_gpu, sort_result, to_device
from test_gpu_parity import _data

pytestmark = pytest.mark.gpu


def _expected(keys, cols, col):
    """(group keys, expected AVG, allowed error or None when bit-exact)."""
    ok, (s, c) = O.groupby(keys, cols, [("sum", col), ("count", None)], nthreads=8)
    if s.dtype == np.float64:
        _, (a,) = O.groupby(keys, cols, [("sumabs", col)], nthreads=8)
        avg = s / c.astype(np.float64)
        return ok, avg, fp_bound(avg, a / c.astype(np.float64), c)
    return ok, s.astype(np.float64) / c.astype(np.float64), None


@pytest.mark.parametrize("strategy", ["table", "partition"])
@pytest.mark.parametrize("kdt", [np.int32, np.int64])
def test_avg_matches_oracle(ctx, strategy, kdt):
    keys, cols = _data(200_003, kdt, 20_000, seed=9, zipf=0.7 if kdt == np.int64 else 0.0)
    aggs = [("avg", 0), ("sum", 2), ("avg", 2), ("avg", 1), ("max", 0)]  # no COUNT: one is added
    gk, ga, res = run_gpu(ctx, keys, cols, aggs, knobs=dict(strategy=strategy))
    gk, ga = sort_result(gk, ga, False)
    for ai, col in ((0, 0), (2, 2), (3, 1)):
        ok, avg, bound = _expected(keys, cols, col)
        np.testing.assert_array_equal(gk, ok)
        assert ga[ai].dtype == np.float64
        if bound is None:
            np.testing.assert_array_equal(ga[ai], avg, err_msg=f"avg of column {col}")
        else:
            assert (np.abs(ga[ai] - avg) <= bound).all(), f"avg of fp32 column {col}"
    ok, (s2, mx) = O.groupby(keys, cols, [("sum", 2), ("max", 0)], nthreads=8)
    np.testing.assert_array_equal(ga[1], s2)
    np.testing.assert_array_equal(ga[4], mx)


def test_avg_with_count_and_learned_sizing(ctx):
    if not E.load_default(ctx):
        pytest.skip("no estimator weights")
    keys, cols = _data(300_000, np.int64, 50_000, seed=4)
    aggs = [("count", None), ("avg", 2)]
    gk, ga, res = run_gpu(ctx, keys, cols, aggs, knobs=dict(sizing="learned", learned_min_rows=-1))
    assert res.stats["predicted_groups"] > 0
    gk, ga = sort_result(gk, ga, False)
    ok, avg, _ = _expected(keys, cols, 2)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(ga[1], avg)
    _, (c,) = O.groupby(keys, cols, [("count", None)], nthreads=8)
    np.testing.assert_array_equal(ga[0], c)


def test_avg_in_batch(ctx):
    """gba_groupby_batch: queries with AVG (with and without their own COUNT)
    beside queries without one, int32 and int64 keys, small and large
    cardinalities; every AVG against the oracle, every other aggregate exact."""
    specs = [  # (rows, key dtype, distinct keys, seed, aggs)
        (50_000, np.int32, 300, 1, [("avg", 0), ("sum", 1)]),
        (120_000, np.int64, 40_000, 2, [("count", None), ("avg", 2), ("min", 0)]),
        (30_000, np.int64, 50, 3, [("sum", 1), ("max", 2)]),
        (80_000, np.int32, 70_000, 4, [("avg", 1), ("avg", 2), ("avg", 0)]),
        (1_000, np.int64, 1_000, 5, [("avg", 2)]),
    ]
    host = [(_data(n, kdt, ndv, seed=sd), aggs) for n, kdt, ndv, sd, aggs in specs]
    qs = [(to_device(k), [to_device(c) for c in cols], aggs) for (k, cols), aggs in host]
    res = ctx.groupby_batch(qs)
    for qi, (((keys, cols), aggs), r) in enumerate(zip(host, res)):
        gk, ga = sort_result(r.keys.cpu().numpy(), [t.cpu().numpy() for t in r.aggs], False)
        for ai, (op, col) in enumerate(aggs):
            msg = f"query {qi} aggregate {ai} ({op})"
            if op == "avg":
                ok, avg, bound = _expected(keys, cols, col)
                np.testing.assert_array_equal(gk, ok, err_msg=msg)
                assert ga[ai].dtype == np.float64, msg
                if bound is None:
                    np.testing.assert_array_equal(ga[ai], avg, err_msg=msg)
                else:
                    assert (np.abs(ga[ai] - avg) <= bound).all(), msg
            else:
                ok, (e,) = O.groupby(keys, cols, [(op, col)], nthreads=8)
                np.testing.assert_array_equal(gk, ok, err_msg=msg)
                if e.dtype == np.float64:
                    _, (a, cnt) = O.groupby(keys, cols, [("sumabs", col), ("count", None)], nthreads=8)
                    assert (np.abs(ga[ai] - e) <= fp_bound(e, a, cnt)).all(), msg
                else:
                    np.testing.assert_array_equal(ga[ai], e, err_msg=msg)
