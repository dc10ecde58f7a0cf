"""Sharded GROUP BY on the library's device steps (one GPU).

Two or three ranks are emulated in one process, without collectives: each
shard is pre-aggregated in key order with the library's kernels, cut into the
owners' runs by the global key range (what the all-reduce gives), owner p's
runs of every shard are concatenated (what the all-to-all delivers), and each
owner merges them.  Kernels of different ranks never wait on one another.  A
world-size-1 NCCL group then runs groupby_sharded end to end, all-to-all
included.  Expected: the oracle over all rows, each key on exactly one owner;
integer aggregates bit-exact, AVG of an integer column exact, fp32 SUM within
the fp32-SUM tolerance."""
import os

import numpy as np
import pytest

import cpu_oracle as O
from cpu_gpu_coprocess_groupby_agg_b200.sharded import (DeviceOps, groupby_sharded, key_range, merge_partials,
                                                        owner_counts, plan_partials, range_cuts)
from gpu_util import fp_bound, to_device

pytestmark = pytest.mark.gpu

AGGS = [("sum", 0), ("count", None), ("min", 0), ("max", 0), ("avg", 0), ("sum", 1), ("avg", 1)]


def _data(n, kdt, ndv, seed):
    rng = np.random.default_rng(seed)
    info = np.iinfo(kdt)
    dom = rng.integers(int(info.min), int(info.max) + 1, size=ndv, dtype=np.int64).astype(kdt)
    keys = dom[rng.integers(0, ndv, size=n)]
    cols = [rng.integers(-(1 << 30), 1 << 30, size=n, dtype=np.int64), rng.standard_normal(n).astype(np.float32)]
    return keys, cols


def _check(gk, ga, keys, cols, label):
    order = np.argsort(gk, kind="stable")
    gk, ga = gk[order], [a[order] for a in ga]
    ek, (s0, c, mn, mx, s1, a1) = O.groupby(keys, cols, [("sum", 0), ("count", None), ("min", 0), ("max", 0),
                                                        ("sum", 1), ("sumabs", 1)], nthreads=8)
    np.testing.assert_array_equal(gk, ek, err_msg=label)
    for g, e in zip(ga[:4], (s0, c, mn, mx)):
        np.testing.assert_array_equal(g, e, err_msg=label)
    np.testing.assert_array_equal(ga[4], s0.astype(np.float64) / c, err_msg=label)
    assert (np.abs(ga[5] - s1) <= fp_bound(s1, a1, c)).all(), label
    assert (np.abs(ga[6] - s1 / c) <= fp_bound(s1 / c, a1 / c, c)).all(), label


@pytest.mark.parametrize("kdt", [np.int32, np.int64, np.uint32])
@pytest.mark.parametrize("nranks", [2, 3])
def test_sharded_steps_emulated(ctx, kdt, nranks):
    import torch
    keys, cols = _data(300_000, kdt, 80_000, seed=7)
    unsigned = kdt == np.uint32
    ops = DeviceOps(ctx)
    plan = plan_partials(AGGS)
    shards = []
    for r in range(nranks):
        k, a = ops.local(to_device(keys[r::nranks].copy()), [to_device(c[r::nranks].copy()) for c in cols],
                         plan.partials, unsigned_keys=unsigned)
        shards.append((k, a))
    ranges = [key_range(k, unsigned) for k, _ in shards]  # what the all-reduce computes
    cuts = range_cuts(min(r[0] for r in ranges), max(r[1] for r in ranges), nranks)
    runs = []
    for k, a in shards:
        counts = owner_counts(k, cuts, unsigned)
        assert len(counts) == nranks and sum(counts) == len(k)
        runs.append((k, a, np.concatenate([[0], np.cumsum(counts)])))
    owned = []
    for p in range(nranks):  # what owner p receives from every shard
        rk = torch.cat([k[off[p]:off[p + 1]] for k, _, off in runs])
        rc = [torch.cat([a[i][off[p]:off[p + 1]] for _, a, off in runs]) for i in range(len(plan.partials))]
        fk, fa = merge_partials(ops, rk, rc, plan, unsigned)
        gk = fk.cpu().numpy()
        owned.append((gk.view(np.uint32) if unsigned else gk, [x.cpu().numpy() for x in fa]))
        assert len(gk) > 0, f"owner {p} got no groups"
    allk = np.concatenate([k for k, _ in owned])
    assert len(np.unique(allk)) == len(allk), "a key on two owners"
    _check(allk, [np.concatenate([a[i] for _, a in owned]) for i in range(len(AGGS))], keys, cols,
           f"{nranks} owners")


def test_sharded_nccl_world_one(ctx):
    import torch
    import torch.distributed as dist
    keys, cols = _data(200_000, np.int64, 30_000, seed=2)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{27000 + os.getpid() % 1000}", rank=0,
                            world_size=1)
    try:
        r = groupby_sharded(ctx, to_device(keys), [to_device(c) for c in cols], AGGS)
        torch.cuda.synchronize()
        _check(r.keys.cpu().numpy(), [a.cpu().numpy() for a in r.aggs], keys, cols, "nccl world 1")
    finally:
        dist.destroy_process_group()
