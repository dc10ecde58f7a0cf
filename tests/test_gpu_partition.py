"""Parity of the radix-partition strategy (histogram -> lookback scan -> staged
scatter -> per-partition shared tables) with the oracle, on the GPU."""
import numpy as np
import pytest

from gpu_util import compare, run_gpu
from test_gpu_parity import AGGS_ALL, _data

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kdt", [np.int32, np.uint32, np.int64])
@pytest.mark.parametrize("bits", [1, 6, 10, 13])
def test_partition_passes(ctx, kdt, bits):
    # about 1,000 groups per partition, so the requested fan-out needs no retry
    keys, cols = _data(700_001, kdt, min(250_000, 1000 << bits), seed=bits)
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=dict(strategy="partition", partition_bits=bits))
    assert res.stats["strategy"] == 2 and res.stats["partition_bits"] == bits
    compare(gk, ga, keys, cols, AGGS_ALL, f"partition {kdt.__name__} bits={bits}")


@pytest.mark.parametrize("n", [0, 1, 5, 2049, 65_537])
def test_partition_tiny_inputs(ctx, n):
    keys, cols = _data(n, np.int64, 1000, seed=n)
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=dict(strategy="partition", partition_bits=3))
    compare(gk, ga, keys, cols, AGGS_ALL, f"partition n={n}")


def test_partition_skew_and_sentinel(ctx):
    keys, cols = _data(1 << 20, np.int64, 300_000, seed=3, zipf=1.2)
    keys[::11] = -1  # all-ones key
    keys[5::13] = np.iinfo(np.int64).min
    gk, ga, _ = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=dict(strategy="partition"))
    compare(gk, ga, keys, cols, AGGS_ALL, "partition skew")
    k32 = keys.astype(np.uint32)
    gk, ga, _ = run_gpu(ctx, k32, cols, AGGS_ALL, knobs=dict(strategy="partition", partition_bits=5))
    compare(gk, ga, k32, cols, AGGS_ALL, "partition skew u32")


def test_partition_fallback_and_retry(ctx):
    """Tiny shared tables force rows into the HBM fallback table; when that
    overflows too the host retries with more partition bits."""
    keys, cols = _data(400_000, np.int64, 300_000, seed=12)
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL,
                          knobs=dict(strategy="partition", partition_bits=4, smem_slots=256))
    compare(gk, ga, keys, cols, AGGS_ALL, "partition fallback")
    assert res.stats["regrows"] >= 1


def test_partition_host_path(ctx):
    keys, cols = _data(2_000_003, np.int64, 900_000, seed=21)
    res = ctx.groupby_host(keys, cols, AGGS_ALL, knobs=dict(strategy="partition"))
    compare(res.keys, res.aggs, keys, cols, AGGS_ALL, "partition host")


def test_auto_strategy_picks_partition_for_high_cardinality(ctx):
    from cpu_gpu_coprocess_groupby_agg_b200 import gen_host
    from cpu_gpu_coprocess_groupby_agg_b200 import workloads as W
    w = W.high_card(n=1 << 23, ndv=1 << 21)
    keys, cols = gen_host(w.spec, w.n)
    gk, ga, res = run_gpu(ctx, keys, cols, w.aggs)
    assert res.stats["strategy"] == 2
    compare(gk, ga, keys, cols, w.aggs, w.name)


@pytest.mark.parametrize("bits", [4, 8])
def test_partition_split_hot_partitions(ctx, bits):
    """Partitions holding hot keys (far more rows than one CTA should take) are
    split into pieces whose groups merge through the HBM table; the all-ones
    key is among the hot ones."""
    keys, cols = _data(1 << 21, np.int64, 2000, seed=40 + bits, zipf=1.5)
    keys[::3] = -1
    gk, ga, res = run_gpu(ctx, keys, cols, AGGS_ALL, knobs=dict(strategy="partition", partition_bits=bits))
    assert res.stats["strategy"] == 2
    compare(gk, ga, keys, cols, AGGS_ALL, f"partition split bits={bits}")
    k32 = keys.astype(np.uint32)
    gk, ga, _ = run_gpu(ctx, k32, cols, AGGS_ALL, knobs=dict(strategy="partition", partition_bits=bits))
    compare(gk, ga, k32, cols, AGGS_ALL, f"partition split u32 bits={bits}")
