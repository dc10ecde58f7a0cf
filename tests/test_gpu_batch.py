"""Parity of the batched path (gba_groupby_batch: work-queue persistent launch,
graph replay, per-query reruns, partition-strategy members) with the oracle."""
import numpy as np
import pytest

from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E
from gpu_util import compare, to_device
from test_gpu_parity import AGGS_ALL, _data

pytestmark = pytest.mark.gpu

AGG_SETS = [
    [("sum", 0), ("count", None)],
    [("count", None)],
    AGGS_ALL,
    [("sum", 2), ("count", None)],
    [("sum", 3)],
    [("min", 0), ("max", 0), ("sum", 1)],
    [("sum", 0), ("sum", 2), ("count", None)],
]


def _queries(count, seed, max_n=150_000):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(0, max_n)) if i % 9 else int(rng.integers(0, 5))
        kdt = [np.int32, np.uint32, np.int64][i % 3]
        ndv = int(max(1, min(n // 2 + 1, 10 ** rng.uniform(0, 5))))
        keys, cols = _data(n, kdt, ndv, seed=seed * 1000 + i, zipf=float(rng.uniform(0, 1.5)))
        out.append((keys, cols, AGG_SETS[i % len(AGG_SETS)]))
    return out


def _device(qs):
    dq = []
    for keys, cols, aggs in qs:
        dq.append((to_device(keys), [to_device(c) for c in cols], aggs, keys.dtype == np.uint32,
                   [c.dtype == np.uint32 for c in cols]))
    return dq


def _check(qs, res, label):
    assert len(res) == len(qs)
    for i, ((keys, cols, aggs), r) in enumerate(zip(qs, res)):
        gk = r.keys.cpu().numpy()
        if keys.dtype == np.uint32:
            gk = gk.view(np.uint32)
        compare(gk, [a.cpu().numpy() for a in r.aggs], keys, cols, aggs, f"{label} query {i}")


@pytest.mark.parametrize("sizing", ["plain", "learned"])
def test_batch_matches_oracle(ctx, sizing):
    if sizing == "learned":
        assert E.load_default(ctx), "committed estimator weights are missing"
    qs = _queries(40, seed=1 if sizing == "plain" else 2)
    res = ctx.groupby_batch(_device(qs), knobs=dict(sizing=sizing))
    _check(qs, res, sizing)


def test_batch_graph_replay_and_direct_launch_agree(ctx):
    qs1 = _queries(24, seed=5)
    # same shapes, new data: the second call replays the captured graph
    qs2 = []
    for i, (keys, cols, aggs) in enumerate(qs1):
        rng = np.random.default_rng(900 + i)
        perm = rng.permutation(len(keys))
        qs2.append((keys[perm].copy(), [c[perm].copy() for c in cols], aggs))
    d1, d2 = _device(qs1), _device(qs2)
    outs = ctx.batch_outputs(d1)
    _check(qs1, ctx.groupby_batch(d1, outs=outs), "graph first")
    _check(qs2, ctx.groupby_batch(d2, outs=outs), "graph replay")
    _check(qs1, ctx.groupby_batch(d1, knobs=dict(use_graph=0)), "direct")


@pytest.mark.parametrize("knobs", [dict(tile_rows=2048), dict(blocks_per_sm=2), dict(item_rows=4096),
                                   dict(smem_slots=128), dict(preagg=0), dict(smem_probe_cap=1),
                                   dict(use_tma=0), dict(use_tma=0, blocks_per_sm=4), dict(nstages=1),
                                   dict(nstages=2), dict(nstages=4), dict(coalesce=1), dict(coalesce=0),
                                   dict(coalesce=1, smem_slots=64), dict(sizing="grow"),
                                   dict(sizing="grow", table_slots=256), dict(use_tma=1, block_threads=512),
                                   dict(use_tma=1, block_threads=1024, nstages=4, coalesce=1),
                                   dict(sizing="learned", block_threads=512)])
def test_batch_knobs_do_not_change_results(ctx, knobs):
    qs = _queries(12, seed=7)
    _check(qs, ctx.groupby_batch(_device(qs), knobs=knobs), str(knobs))


def test_batch_overflow_reruns_query_alone(ctx):
    qs = _queries(10, seed=9)
    res = ctx.groupby_batch(_device(qs), knobs=dict(sizing="fixed", table_slots=64, probe_cap=16, max_regrow=8,
                                                      strategy="table"))
    _check(qs, res, "overflow")
    assert res[0].stats["regrows"] >= 1


def test_batch_with_partition_members(ctx):
    qs = _queries(6, seed=11)
    # plain sizing at load 0.055: 4M rows -> 2^27 slots, a 3.2 GB table, past the batch's
    # 2 GB bound -> partition; the small queries stay on the table strategy
    keys, cols = _data(4_000_000, np.int64, 2_000_000, seed=99)
    qs.insert(3, (keys, cols, [("sum", 0), ("count", None)]))
    res = ctx.groupby_batch(_device(qs), knobs=dict(load_factor=0.055))
    _check(qs, res, "mixed strategies")
    assert res[0].stats["strategy"] == A.STRATEGY_AUTO  # both kinds ran


def test_batch_empty_and_capacity_error(ctx):
    assert ctx.groupby_batch([]) == []
    qs = _queries(3, seed=13)
    keys, cols = _data(10_000, np.int64, 5000, seed=1)
    qs.append((keys, cols, [("count", None)]))
    dq = _device(qs)
    outs = ctx.batch_outputs(dq, capacity=[len(q[0]) + 1 for q in qs[:-1]] + [10])
    with pytest.raises(A.GbaError) as e:
        ctx.groupby_batch(dq, outs=outs)
    assert e.value.status == A.ERR_OUTPUT_CAPACITY


def test_batch_bulk_copy_kernel_ragged_and_unaligned(ctx):
    """The bulk-copy kernel's edges: queries whose row count is not a multiple
    of 4 (tail rows read from global memory), fewer rows than one stage, one
    row, and columns that start off a 16-byte boundary (no bulk copies)."""
    import torch
    qs = []
    for i, n in enumerate([1, 3, 5, 2047, 2049, 4099, 70_001, 131_075]):
        keys, cols = _data(n, [np.int32, np.int64][i % 2], max(1, n // 7), seed=300 + i, zipf=1.2)
        qs.append((keys, cols, [("sum", 0), ("count", None), ("min", 0)]))
    dq = _device(qs)
    # a query whose key and value columns start off a 16-byte boundary: 4 and
    # 8 bytes into their buffers
    keys, cols = _data(50_001, np.int32, 3000, seed=333)
    cols = cols[:1]
    kb = torch.zeros(50_002, dtype=torch.int32, device="cuda")
    kb[1:] = torch.from_numpy(keys).cuda()
    vb = torch.zeros(50_002, dtype=torch.int64, device="cuda")
    vb[1:] = torch.from_numpy(cols[0]).cuda()
    qs.append((keys, cols, [("sum", 0), ("count", None), ("min", 0)]))
    dq.append((kb[1:], [vb[1:]], qs[-1][2], False, [False]))
    for knobs in (dict(), dict(coalesce=1), dict(nstages=1), dict(use_tma=1, block_threads=512),
                  dict(use_tma=1, block_threads=1024)):
        _check(qs, ctx.groupby_batch(dq, knobs=knobs), f"ragged {knobs}")


@pytest.mark.parametrize("cluster", [2, 4, 8, 16])
def test_batch_cluster_tables_match_oracle(ctx, cluster):
    """Queries whose predicted groups outgrow one CTA's shared table but fit a
    cluster's (learned sizing, integer SUM/COUNT): their shared table is spread
    over the CTAs of a thread-block cluster (distributed shared memory)."""
    assert E.load_default(ctx), "committed estimator weights are missing"
    specs = [(400_000, np.int64, 12_000, 0.0), (600_000, np.int32, 30_000, 0.3), (300_000, np.uint32, 60_000, 0.0),
             (900_000, np.int64, 100_000, 0.8), (250_000, np.int32, 8_000, 1.1), (50_000, np.int64, 200, 0.5)]
    aggsets = [[("sum", 0), ("count", None)], [("count", None)], [("sum", 0), ("sum", 2), ("count", None)],
               [("sum", 3), ("count", None)], [("sum", 0), ("count", None)], [("sum", 0), ("count", None)]]
    qs = []
    for i, ((n, kdt, ndv, z), aggs) in enumerate(zip(specs, aggsets)):
        keys, cols = _data(n, kdt, ndv, seed=700 + i, zipf=z)
        qs.append((keys, cols, aggs))
    res = ctx.groupby_batch(_device(qs), knobs=dict(sizing="learned", cluster_ctas=cluster))
    _check(qs, res, f"cluster {cluster}")
    # the same with the graph replayed and with warp combining forced
    res = ctx.groupby_batch(_device(qs), knobs=dict(sizing="learned", cluster_ctas=cluster, coalesce=1))
    _check(qs, res, f"cluster {cluster} combined")


@pytest.mark.parametrize("knobs", [dict(exchange=1), dict(exchange=1, sizing="learned"),
                                   dict(exchange=1, smem_probe_cap=1)])
def test_batch_owner_exchange_matches_oracle(ctx, knobs):
    """Every table query through the owner-exchange kernel (each SM owns a
    range of keys; rows reach their owner through buffers that alternate
    between windows): all key types and aggregate signatures of the mixed
    queries, empty and tiny queries among them."""
    if knobs.get("sizing") == "learned":
        assert E.load_default(ctx), "committed estimator weights are missing"
    qs = _queries(20, seed=21)
    _check(qs, ctx.groupby_batch(_device(qs), knobs=knobs), str(knobs))


def test_batch_owner_exchange_windows_and_overflow(ctx):
    """Queries longer than one exchange window (2^20 rows), groups beyond the
    SMs' shared tables (keys go to the HBM table, each key in one place), and
    the automatic choice under learned sizing."""
    assert E.load_default(ctx), "committed estimator weights are missing"
    specs = [(2_500_003, np.int64, 300_000, 0.0), (1_200_000, np.int32, 40_000, 0.2),
             (1_500_000, np.uint32, 2_000_000, 0.0), (700_000, np.int64, 20_000, 0.4)]
    aggsets = [[("sum", 0), ("count", None)], [("sum", 0), ("sum", 2), ("count", None)],
               [("sum", 3), ("count", None)], AGGS_ALL]
    qs = []
    for i, ((n, kdt, ndv, z), aggs) in enumerate(zip(specs, aggsets)):
        keys, cols = _data(n, kdt, ndv, seed=800 + i, zipf=z)
        qs.append((keys, cols, aggs))
    for knobs in (dict(exchange=1), dict(sizing="learned"), dict(sizing="learned", exchange=0)):
        _check(qs, ctx.groupby_batch(_device(qs), knobs=knobs), f"exchange {knobs}")


def test_batch_owner_exchange_on_the_batch_class_256_4096(ctx):
    """The 86 queries of the benchmark batch with 256 to 4095 distinct ids
    (Zipf s in [0, 1.5]), every one forced through the owner-exchange kernel
    with hot tables where the sample is skewed: the case that once exposed
    hot-table partial records written over the other exchange buffer."""
    import torch
    from cpu_gpu_coprocess_groupby_agg_b200 import gen_device, workloads as W
    assert E.load_default(ctx), "committed estimator weights are missing"
    allq = [q for q in W.batch_queries() if 256 <= q.meta["ndv"] < 4096]
    dq = [(*gen_device(q.spec, q.n), q.aggs) for q in allq]
    res = ctx.groupby_batch(dq, knobs=dict(sizing="learned", exchange=1))
    for q, (k, c, _), r in zip(allq, dq, res):
        order = torch.argsort(r.keys)
        gk = r.keys[order].cpu().numpy()
        ga = [a[order].cpu().numpy() for a in r.aggs]
        compare(gk, ga, k.cpu().numpy(), [x.cpu().numpy() for x in c], q.aggs, label=q.name, presorted=True)


def _host_outs(qs, pinned=True):
    import torch
    from cpu_gpu_coprocess_groupby_agg_b200 import _abi as AB
    from cpu_gpu_coprocess_groupby_agg_b200.api import agg_is_fp, parse_aggs, _np_type

    def buf(n, dt):
        if not pinned:
            return np.empty(n, dtype=dt)
        t = torch.empty(n * np.dtype(dt).itemsize, dtype=torch.uint8).pin_memory()
        return t.numpy().view(dt)

    outs = []
    for keys, cols, aggs in qs:
        cap = max(len(keys), 1) + 1
        oaggs = [buf(cap, np.float64 if (op != AB.COUNT and agg_is_fp(op, _np_type(cols[c]))) else np.int64)
                 for op, c in parse_aggs(aggs)]
        outs.append((buf(cap, keys.dtype), oaggs))
    return outs


@pytest.mark.parametrize("knobs", [dict(), dict(sizing="learned")])
def test_batch_host_matches_oracle(ctx, knobs):
    """gba_groupby_batch_host: host columns in, host buffers out, the queries
    cut into parts whose copies overlap the previous part's aggregation."""
    if knobs.get("sizing") == "learned" and not E.load_default(ctx):
        pytest.skip("no estimator weights")
    qs = _queries(14, seed=21, max_n=400_000)
    # two large queries, so that the batch spans several parts of >= 64 MB
    for j in range(2):
        keys, cols = _data(3_000_000 + j, [np.int64, np.uint32][j], 200_000, seed=77 + j, zipf=0.6)
        qs.insert(5 * j + 2, (keys, cols, AGGS_ALL))
    res = ctx.groupby_batch_host(qs, _host_outs(qs), knobs=knobs)
    for i, ((keys, cols, aggs), r) in enumerate(zip(qs, res)):
        compare(r.keys, r.aggs, keys, cols, aggs, f"host batch {knobs} query {i}")


def test_batch_host_pageable_and_empty(ctx):
    """Pageable host buffers, empty queries and a batch of one."""
    qs = _queries(5, seed=23, max_n=20_000)
    qs.append((np.zeros(0, dtype=np.int64), _data(0, np.int64, 1)[1], [("count", None)]))
    res = ctx.groupby_batch_host(qs, _host_outs(qs, pinned=False))
    for i, ((keys, cols, aggs), r) in enumerate(zip(qs, res)):
        compare(r.keys, r.aggs, keys, cols, aggs, f"pageable query {i}")
    assert ctx.groupby_batch_host([], []) == []
    one = qs[:1]
    r = ctx.groupby_batch_host(one, _host_outs(one))[0]
    compare(r.keys, r.aggs, *one[0], "batch of one")

