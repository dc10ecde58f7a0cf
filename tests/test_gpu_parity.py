"""Parity of the CUDA path (through the C ABI) with the oracle, on the GPU."""
import numpy as np
import pytest

from cpu_gpu_coprocess_groupby_agg_b200 import gen_host, make_knobs
from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
from cpu_gpu_coprocess_groupby_agg_b200 import workloads as W
from gpu_util import compare, run_gpu

pytestmark = pytest.mark.gpu

AGGS_ALL = [("sum", 0), ("count", None), ("min", 0), ("max", 0), ("sum", 1), ("sum", 2), ("min", 2), ("max", 3)]


def _data(n, kdt, ndv, seed=0, zipf=0.0):
    rng = np.random.default_rng(seed)
    if zipf > 0:
        ranks = np.minimum(rng.zipf(1.0 + zipf, size=n), ndv) - 1
    else:
        ranks = rng.integers(0, ndv, size=n)
    if kdt == np.int64:
        dom = rng.integers(-(1 << 62), 1 << 62, size=ndv, dtype=np.int64)
    else:
        info = np.iinfo(kdt)
        dom = rng.integers(int(info.min), int(info.max) + 1, size=ndv, dtype=np.int64).astype(kdt)
    keys = dom[ranks]
    cols = [rng.integers(-(1 << 40), 1 << 40, size=n, dtype=np.int64),
            rng.standard_normal(n).astype(np.float32),
            rng.integers(-1000, 1000, size=n, dtype=np.int32).astype(np.int32),
            rng.integers(0, 1 << 32, size=n, dtype=np.int64).astype(np.uint32)]
    return keys, cols


@pytest.mark.parametrize("kdt", [np.int32, np.uint32, np.int64])
@pytest.mark.parametrize("ndv", [1, 37, 1024, 20_000, 300_000])
def test_types_and_cardinalities(ctx, kdt, ndv):
    keys, cols = _data(400_003, kdt, ndv, seed=ndv)
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL)
    compare(gk, ga, keys, cols, AGGS_ALL, f"{kdt.__name__}/{ndv}")


@pytest.mark.parametrize("knobs", [
    dict(use_tma=0), dict(use_tma=1), dict(coalesce=0), dict(coalesce=1), dict(preagg=0), dict(smem_slots=64),
    dict(smem_probe_cap=1), dict(tile_rows=512, block_threads=128), dict(nstages=1), dict(blocks_per_sm=2),
    dict(strategy="table"),
])
def test_knobs_do_not_change_results(ctx, knobs):
    keys, cols = _data(1 << 20, np.int64, 5000, seed=3, zipf=1.1)
    gk, ga, _ = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=knobs)
    compare(gk, ga, keys, cols, AGGS_ALL, str(knobs))


@pytest.mark.parametrize("n", [0, 1, 2, 31, 33, 2047, 2049, 4096 * 3 + 5])
def test_ragged_and_tiny(ctx, n):
    keys, cols = _data(n, np.int64, 50, seed=n)
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL)
    assert res.n_groups == len(np.unique(keys))
    compare(gk, ga, keys, cols, AGGS_ALL, f"n={n}")


def test_misaligned_columns_fall_back_from_tma(ctx):
    import torch
    keys, cols = _data(100_001, np.int64, 999, seed=9)
    dk = torch.from_numpy(np.concatenate([[0], keys])).cuda()[1:]  # 8-byte but not 16-byte aligned
    dcols = [torch.from_numpy(np.concatenate([c[:1], c]).view(np.int32 if c.dtype == np.uint32 else c.dtype)).cuda()[1:]
             for c in cols]
    res = ctx.groupby(dk, dcols, AGGS_ALL, unsigned_cols=[False, False, False, True])
    compare(res.keys.cpu().numpy(), [a.cpu().numpy() for a in res.aggs], keys, cols, AGGS_ALL, "misaligned")


def test_sentinel_and_extreme_keys(ctx):
    n = 300_000
    rng = np.random.default_rng(1)
    special64 = np.array([-1, 0, np.iinfo(np.int64).min, np.iinfo(np.int64).max, 1], dtype=np.int64)
    keys = special64[rng.integers(0, 5, size=n)]
    keys[::7] = rng.integers(-100, 100, size=len(keys[::7]))
    cols = [rng.integers(-5, 5, size=n, dtype=np.int64), rng.standard_normal(n).astype(np.float32),
            np.ones(n, dtype=np.int32), np.ones(n, dtype=np.uint32)]
    for kn in (None, dict(preagg=0)):
        gk, ga, _ = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=kn)
        compare(gk, ga, keys, cols, AGGS_ALL, f"sentinel64 {kn}")
    keys32 = np.array([0xFFFFFFFF, 0, 0x80000000, 5], dtype=np.uint32)[rng.integers(0, 4, size=n)]
    gk, ga, _ = run_gpu(ctx, keys32, cols, AGGS_ALL)
    compare(gk, ga, keys32, cols, AGGS_ALL, "sentinel u32")
    keys_i32 = keys32.view(np.int32)
    gk, ga, _ = run_gpu(ctx, keys_i32, cols, AGGS_ALL, knobs=dict(preagg=0))
    compare(gk, ga, keys_i32, cols, AGGS_ALL, "sentinel i32")


def test_regrow_on_overflow(ctx):
    keys, cols = _data(200_000, np.int64, 150_000, seed=4)
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL,
                          knobs=dict(sizing="fixed", table_slots=1024, probe_cap=32, max_regrow=6, strategy="table"))
    assert res.stats["regrows"] >= 1
    compare(gk, ga, keys, cols, AGGS_ALL, "regrow")


def test_overflow_limit_reports_error(ctx):
    keys, cols = _data(50_000, np.int64, 40_000, seed=5)
    with pytest.raises(A.GbaError) as e:
        run_gpu(ctx, keys, cols, AGGS_ALL, knobs=dict(sizing="fixed", table_slots=256, probe_cap=4, max_regrow=0))
    assert e.value.status == A.ERR_TABLE_OVERFLOW


def test_output_capacity_error(ctx):
    keys, cols = _data(10_000, np.int64, 500, seed=6)
    with pytest.raises(A.GbaError) as e:
        run_gpu(ctx, keys, cols, AGGS_ALL, capacity=100)
    assert e.value.status == A.ERR_OUTPUT_CAPACITY


def test_small_workload_vs_oracle(ctx):
    w = W.small()
    keys, cols = gen_host(w.spec, w.n, key_unsigned=True)
    gk, ga, res = run_gpu(ctx, keys, cols, w.aggs)
    assert res.n_groups == 1024
    compare(gk, ga, keys, cols, w.aggs, w.name)


def test_host_resident_path(ctx):
    keys, cols = _data(3_000_017, np.int64, 70_000, seed=8, zipf=0.9)
    res = ctx.groupby_host(keys, cols, AGGS_ALL)
    compare(res.keys, res.aggs, keys, cols, AGGS_ALL, "host")
    keys32, cols32 = _data(123_457, np.uint32, 2000, seed=2)
    res = ctx.groupby_host(keys32, cols32, AGGS_ALL, knobs=dict(use_tma=0))
    compare(res.keys, res.aggs, keys32, cols32, AGGS_ALL, "host u32")


def test_repeat_calls_identical(ctx):
    keys, cols = _data(1 << 20, np.int64, 10_000, seed=10, zipf=1.2)
    first = run_gpu(ctx, keys, cols, AGGS_ALL)
    for _ in range(3):
        again = run_gpu(ctx, keys, cols, AGGS_ALL)
        compare(again[0], again[1], keys, cols, AGGS_ALL, "repeat")
    assert first[2].n_groups == again[2].n_groups
