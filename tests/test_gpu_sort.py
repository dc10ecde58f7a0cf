"""Key-ordered output (gba_knobs.sort_output): the groups come back in
ascending key order (signed for int32/int64 keys, unsigned for u32) with every
aggregate permuted alike.  The oracle's output is sorted by key, so the CUDA
result is compared element by element with no sort on the test's side: keys
and integer aggregates bit-exact, fp32 SUM within the fp32-SUM tolerance.
Covered: the three key types, the table and partition strategies, the batch
and host-resident entry points, AVG, zero and one group, the extreme keys
(the all-ones key, INT_MIN, INT_MAX) and a multi-million-group case that runs
every radix pass."""
import numpy as np
import pytest

import cpu_oracle as O
from gpu_util import fp_bound, run_gpu, to_device
from test_gpu_parity import _data

pytestmark = pytest.mark.gpu

AGGS = [("sum", 0), ("count", None), ("min", 2), ("max", 3), ("sum", 1)]


def _check_ordered(gk, ga, keys, cols, aggs, label):
    ok, oa = O.groupby(keys, cols, aggs, nthreads=8)
    assert len(gk) == len(ok), f"{label}: {len(gk)} groups vs oracle {len(ok)}"
    np.testing.assert_array_equal(gk, ok, err_msg=f"{label}: keys out of order or wrong")
    for i, ((op, col), g, o) in enumerate(zip(aggs, ga, oa)):
        if o.dtype == np.float64:
            _, (a, cnt) = O.groupby(keys, cols, [("sumabs", col), ("count", None)], nthreads=8)
            assert (np.abs(g - o) <= fp_bound(o, a, cnt)).all(), f"{label}: agg {i}"
        else:
            np.testing.assert_array_equal(g, o, err_msg=f"{label}: agg {i} ({op})")


@pytest.mark.parametrize("strategy", ["table", "partition"])
@pytest.mark.parametrize("kdt", [np.int32, np.int64, np.uint32])
def test_sorted_output_matches_oracle_order(ctx, strategy, kdt):
    keys, cols = _data(300_007, kdt, 60_000, seed=21, zipf=0.8 if kdt == np.int64 else 0.0)
    gk, ga, _ = run_gpu(ctx, keys, cols, AGGS, knobs=dict(strategy=strategy, sort_output=1))
    _check_ordered(gk, ga, keys, cols, AGGS, f"{strategy} {np.dtype(kdt).name}")


def test_sorted_extreme_keys(ctx):
    rng = np.random.default_rng(3)
    for kdt in (np.int32, np.int64, np.uint32):
        info = np.iinfo(kdt)
        special = np.array([info.min, info.max, info.min + 1, info.max - 1, 0, 1], dtype=kdt)
        if kdt != np.uint32:
            special = np.concatenate([special, np.array([-1, -2], dtype=kdt)])  # -1: the all-ones key
        keys = rng.choice(special, size=50_000).astype(kdt)
        cols = [rng.integers(-1000, 1000, size=50_000, dtype=np.int64)]
        aggs = [("sum", 0), ("count", None)]
        gk, ga, _ = run_gpu(ctx, keys, cols, aggs, knobs=dict(sort_output=1))
        _check_ordered(gk, ga, keys, cols, aggs, f"extremes {np.dtype(kdt).name}")


def test_sorted_zero_and_one_group(ctx):
    cols = [np.arange(1000, dtype=np.int64)]
    keys = np.full(1000, 7, dtype=np.int64)
    gk, ga, _ = run_gpu(ctx, keys, cols, [("sum", 0)], knobs=dict(sort_output=1))
    _check_ordered(gk, ga, keys, cols, [("sum", 0)], "one group")
    e = np.zeros(0, dtype=np.int64)
    gk, ga, res = run_gpu(ctx, e, [e.copy()], [("sum", 0)], knobs=dict(sort_output=1))
    assert res.n_groups == 0 and len(gk) == 0


def test_sorted_many_groups_every_pass(ctx):
    """int64 keys over [-2^62, 2^62): eight 8-bit passes over about 2.65M
    groups (2^22 uniform draws from 2^22 keys; about 650 tiles of the scatter)."""
    keys, cols = _data(1 << 22, np.int64, 1 << 22, seed=8)
    aggs = [("sum", 0), ("count", None)]
    gk, ga, res = run_gpu(ctx, keys, cols, aggs, knobs=dict(sort_output=1))
    assert res.n_groups > 2_500_000
    _check_ordered(gk, ga, keys, cols, aggs, "many groups")


def test_sorted_with_avg(ctx):
    keys, cols = _data(100_000, np.int32, 5_000, seed=2)
    gk, ga, _ = run_gpu(ctx, keys, cols, [("avg", 0), ("count", None)], knobs=dict(sort_output=1))
    ok, (s, c) = O.groupby(keys, cols, [("sum", 0), ("count", None)], nthreads=8)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(ga[0], s.astype(np.float64) / c.astype(np.float64))
    np.testing.assert_array_equal(ga[1], c)


def test_sorted_batch(ctx):
    specs = [(40_000, np.int32, 900, 1), (120_000, np.int64, 80_000, 2), (5_000, np.uint32, 4_000, 3),
             (1, np.int64, 1, 4), (70_000, np.int64, 20, 5)]
    host = [_data(n, kdt, ndv, seed=sd) for n, kdt, ndv, sd in specs]
    aggs = [("sum", 0), ("count", None), ("max", 2)]
    qs = [(to_device(k), [to_device(c) for c in cols], aggs, k.dtype == np.uint32,
           [c.dtype == np.uint32 for c in cols]) for k, cols in host]
    res = ctx.groupby_batch(qs, knobs=dict(sort_output=1))
    for qi, ((keys, cols), r) in enumerate(zip(host, res)):
        gk = r.keys.cpu().numpy()
        if keys.dtype == np.uint32:
            gk = gk.view(np.uint32)
        _check_ordered(gk, [a.cpu().numpy() for a in r.aggs], keys, cols, aggs, f"batch query {qi}")


def test_sorted_host_resident(ctx):
    keys, cols = _data(200_000, np.int64, 30_000, seed=6)
    aggs = [("sum", 0), ("count", None), ("sum", 1)]
    r = ctx.groupby_host(keys, cols, aggs, knobs=dict(sort_output=1))
    _check_ordered(np.asarray(r.keys), [np.asarray(a) for a in r.aggs], keys, cols, aggs, "host-resident")
