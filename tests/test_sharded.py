"""Sharded GROUP BY across ranks on CPU: gloo, world size 2.

The range cuts, owner runs, exchange and merge logic of
cpu_gpu_coprocess_groupby_agg_b200.sharded run for real over gloo all-reduces
and all-to-alls; its device steps (local partial aggregation in key order,
merge, AVG division) are stood in for by the oracle, so that the multi-rank
path is covered without a GPU.  The union of the
ranks' groups must equal the oracle over all rows, with each key on exactly one
rank."""
import os
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

AGGS = [("sum", 0), ("count", None), ("min", 0), ("max", 0), ("avg", 0), ("sum", 1), ("avg", 1)]


class OracleOps:
    """The sharded path's device steps, restated on the CPU oracle."""

    def local(self, keys, cols, partials, unsigned_keys=False, unsigned_cols=(), knobs=None):
        """Partial groups in key order."""
        import torch
        import cpu_oracle as O
        k, outs = O.groupby(keys.numpy(), [c.numpy() for c in cols], list(partials), nthreads=2)
        return torch.from_numpy(k), [torch.from_numpy(o) for o in outs]

    def merge(self, keys, cols, merge_aggs, unsigned_keys=False):
        return self.local(keys, cols, merge_aggs)

    def avg_divide(self, sums, fp, count):
        return [s.double() / count.double() for s in sums]


def _data(seed=5, n=20_000):
    rng = np.random.default_rng(seed)
    dom = rng.integers(-(1 << 50), 1 << 50, size=3_000, dtype=np.int64)
    keys = dom[rng.integers(0, len(dom), size=n)]
    cols = [rng.integers(-(1 << 30), 1 << 30, size=n, dtype=np.int64), rng.standard_normal(n).astype(np.float32)]
    return keys, cols


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from cpu_gpu_coprocess_groupby_agg_b200.sharded import groupby_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    keys, cols = _data()
    mine = slice(rank, None, world)
    r = groupby_sharded(None, torch.from_numpy(keys[mine].copy()), [torch.from_numpy(c[mine].copy()) for c in cols],
                        AGGS, ops=OracleOps())
    q.put((rank, r.keys.numpy(), [a.numpy() for a in r.aggs]))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_groupby_gloo():
    import cpu_oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 28000 + os.getpid() % 1000
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict((r, (k, a)) for r, k, a in (q.get(timeout=120) for _ in range(2)))
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    k0, k1 = got[0][0], got[1][0]
    assert len(np.intersect1d(k0, k1)) == 0, "a key on two ranks"
    assert len(k0) > 0 and len(k1) > 0
    gk = np.concatenate([k0, k1])
    ga = [np.concatenate([got[0][1][i], got[1][1][i]]) for i in range(len(AGGS))]
    order = np.argsort(gk)
    gk, ga = gk[order], [a[order] for a in ga]
    keys, cols = _data()
    ek, (s0, c, mn, mx, s1, a1) = O.groupby(keys, cols, [("sum", 0), ("count", None), ("min", 0), ("max", 0),
                                                        ("sum", 1), ("sumabs", 1)], nthreads=2)
    np.testing.assert_array_equal(gk, ek)
    for g, e in zip(ga[:4], (s0, c, mn, mx)):
        np.testing.assert_array_equal(g, e)
    np.testing.assert_array_equal(ga[4], s0.astype(np.float64) / c)
    assert (np.abs(ga[5] - s1) <= 1e-6 * np.abs(s1) + 1e-12 * a1).all()
    assert (np.abs(ga[6] - s1 / c) <= 1e-6 * np.abs(s1 / c) + 1e-12 * a1 / c).all()


def test_range_cuts_and_owner_runs():
    """The range cuts split [lo, hi] into nparts nonempty ranges that cover it;
    the owner runs of a key-ordered shard follow them, u32 keys read unsigned."""
    import torch
    from cpu_gpu_coprocess_groupby_agg_b200.sharded import key_range, owner_counts, range_cuts
    for lo, hi, p in [(0, 0, 1), (5, 5, 4), (-10, 10, 3), (-(1 << 63), (1 << 63) - 1, 8), (0, (1 << 32) - 1, 5)]:
        cuts = range_cuts(lo, hi, p)
        assert len(cuts) == p - 1
        edges = [lo] + cuts + [hi + 1]
        assert all(a <= b for a, b in zip(edges, edges[1:])) and edges[0] == lo and edges[-1] == hi + 1
        if hi - lo + 1 >= p:
            assert all(a < b for a, b in zip(edges, edges[1:])), (lo, hi, p)
    # a key-ordered shard of signed keys
    k = torch.tensor([-9, -3, 0, 2, 7, 10], dtype=torch.int64)
    assert key_range(k) == (-9, 10)
    cuts = range_cuts(-10, 10, 3)  # owners own [-10,-3), [-3,4), [4,10]
    assert owner_counts(k, cuts) == [1, 3, 2]
    # u32 keys held in an int32 tensor, in unsigned order (0x80000000 and up last)
    u = torch.tensor([1, 2, 0x7FFFFFFF, -0x80000000, -1], dtype=torch.int32)
    assert key_range(u, True) == (1, 0xFFFFFFFF)
    assert owner_counts(u, range_cuts(0, 0xFFFFFFFF, 2), True) == [3, 2]
    # an empty shard still reports one run per owner
    assert key_range(torch.empty(0, dtype=torch.int64)) is None
    assert owner_counts(torch.empty(0, dtype=torch.int64), [1, 2]) == [0, 0, 0]


def test_plan_partials_shares_partials():
    """AVG becomes SUM and COUNT partials shared with the caller's own SUM and
    COUNT; ops without a partial merge are refused."""
    import pytest
    from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
    from cpu_gpu_coprocess_groupby_agg_b200.sharded import plan_partials
    p = plan_partials([("sum", 0), ("avg", 0), ("count", None), ("avg", 1), ("max", 1)])
    assert p.partials == [(A.SUM, 0), (A.COUNT, 0), (A.SUM, 1), (A.MAX, 1)]
    assert p.final == [("col", 0), ("avg", 0, 1), ("col", 1), ("avg", 2, 1), ("col", 3)]
    with pytest.raises(ValueError):
        plan_partials([("count_valid", 0)])
