"""Sharded GROUP BY across ranks: one process per GPU, torch.distributed for
the exchange (NCCL over NVLink under the ``nccl`` backend).

Each rank holds a shard of the rows; the result is distributed: every group
lives on exactly one rank (its owner), and each rank gets back the groups it
owns, in key order.  Owners own key ranges: the range between the smallest and
the largest key of all ranks (one all-reduce) cut into equal parts.  Per rank:

1. local partial aggregation of the shard in key order (``gba_groupby`` with
   ``sort_output``): AVG becomes a SUM and a COUNT, every other aggregate its
   own partial;
2. each owner's run of the sorted partial groups found by a binary search of
   the range cuts;
3. one all-to-all of the run lengths, then one all-to-all per column;
4. the owner merges what it received (``gba_groupby`` in key order: SUM of the
   SUMs and COUNTs, MIN of the MINs, MAX of the MAXes, partial columns in
   groups of at most four whose outputs align because the keys are sorted)
   and divides the AVGs (``gba_avg_divide``).

Equal cuts of the key range balance keys spread over it; keys bunched in a
narrow part of their range load a few owners more.  No reference counterpart:
the reference runs on one device (test/test.cu:35).  The exchange is NCCL's
all-to-all, not a kernel of this library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

from . import _abi as A
from .api import Result, parse_aggs

_MERGE = {A.SUM: A.SUM, A.COUNT: A.SUM, A.MIN: A.MIN, A.MAX: A.MAX}


@dataclass
class PartialPlan:
    partials: list          # [(op, col)] of the local query
    final: list             # per caller aggregate: ("col", i) or ("avg", sum_i, count_i)


def plan_partials(aggs: Sequence) -> PartialPlan:
    """The local query's partial aggregates and how each caller aggregate is
    read back from the merged partials."""
    partials, final = [], []

    def add(p):
        if p not in partials:
            partials.append(p)
        return partials.index(p)

    for op, col in parse_aggs(aggs):
        if op == A.AVG:
            final.append(("avg", add((A.SUM, col)), add((A.COUNT, 0))))
        elif op in _MERGE:
            final.append(("col", add((op, 0 if op == A.COUNT else col))))
        else:
            raise ValueError("sharded GROUP BY takes SUM, COUNT, MIN, MAX and AVG")
    return PartialPlan(partials, final)


class DeviceOps:
    """The device steps, on the library's kernels."""

    def __init__(self, ctx):
        self.ctx = ctx

    def local(self, keys, cols, partials, unsigned_keys=False, unsigned_cols=(), knobs=None):
        """Partial groups of a shard, in key order."""
        kn = dict(knobs or {}, sort_output=1)
        r = self.ctx.groupby(keys, cols, partials, knobs=kn, unsigned_keys=unsigned_keys, unsigned_cols=unsigned_cols)
        return r.keys, list(r.aggs)

    def merge(self, keys, cols, merge_aggs, unsigned_keys=False):
        r = self.ctx.groupby(keys, cols, merge_aggs, knobs=dict(sort_output=1), unsigned_keys=unsigned_keys)
        return r.keys, list(r.aggs)

    def avg_divide(self, sums, fp, count):
        import torch
        if not sums or count.numel() == 0:
            return [s.view(torch.float64) if s.dtype == torch.int64 else s for s in sums]
        sp = (C.c_void_p * len(sums))(*[s.data_ptr() for s in sums])
        fl = (C.c_int32 * len(sums))(*[int(f) for f in fp])
        s = torch.cuda.current_stream(count.device)
        A.check(self.ctx._lib.gba_avg_divide(self.ctx._h, len(sums), sp, fl, C.c_void_p(count.data_ptr()),
                                             count.numel(), C.c_void_p(s.cuda_stream)), self.ctx._h)
        return [x.view(torch.float64) for x in sums]


def merge_partials(ops, keys, pcols, plan: PartialPlan, unsigned_keys=False):
    """Owner side: merges received partial columns by key; returns (keys, the
    caller's aggregates)."""
    merged = [None] * len(plan.partials)
    out_keys = None
    for lo in range(0, len(plan.partials), A.GBA_MAX_COLS):
        idx = list(range(lo, min(lo + A.GBA_MAX_COLS, len(plan.partials))))
        mk, ma = ops.merge(keys, [pcols[i] for i in idx],
                           [(_MERGE[plan.partials[i][0]], j) for j, i in enumerate(idx)], unsigned_keys)
        if out_keys is None:
            out_keys = mk
        elif len(mk) != len(out_keys):
            raise RuntimeError("merge chunks disagree on the group count")
        for j, i in enumerate(idx):
            merged[i] = ma[j]
    # AVG: SUM / COUNT, one divide per count column
    avg_cols = {}
    for f in plan.final:
        if f[0] == "avg":
            avg_cols.setdefault(f[2], []).append(f[1])
    import torch
    results = {}
    for ci, sis in avg_cols.items():
        sums = [merged[i].clone() for i in sis]  # a SUM may also be a caller's aggregate
        fp = [s.dtype == torch.float64 for s in sums]
        for i, v in zip(sis, ops.avg_divide(sums, fp, merged[ci])):
            results[("avg", i, ci)] = v
    aggs_out = [merged[f[1]] if f[0] == "col" else results[f] for f in plan.final]
    return out_keys, aggs_out


def _order_keys(keys, unsigned_keys):
    """The keys as int64 values whose order is the keys' own (u32 bits read
    unsigned)."""
    import torch
    k = keys.to(torch.int64)
    return k & 0xFFFFFFFF if unsigned_keys else k


def key_range(keys, unsigned_keys=False):
    """(smallest, largest) key of a key-ordered shard, as Python ints (None for
    an empty shard)."""
    if keys.numel() == 0:
        return None
    k = _order_keys(keys[:1], unsigned_keys).item(), _order_keys(keys[-1:], unsigned_keys).item()
    return k


def range_cuts(lo: int, hi: int, nparts: int) -> list:
    """Owner p owns keys in [cut[p-1], cut[p]) (cut[-1] = -inf, cut[nparts-1] = +inf)."""
    span = hi - lo + 1
    return [lo + span * p // nparts for p in range(1, nparts)]


def owner_counts(keys, cuts, unsigned_keys=False) -> list:
    """Lengths of the owners' runs of a key-ordered shard."""
    import torch
    n = keys.numel()
    if n == 0:
        return [0] * (len(cuts) + 1)
    b = torch.searchsorted(_order_keys(keys, unsigned_keys),
                           torch.tensor(cuts, dtype=torch.int64, device=keys.device)).tolist() if cuts else []
    edges = [0] + [int(x) for x in b] + [n]
    return [edges[i + 1] - edges[i] for i in range(len(edges) - 1)]


def global_range(local, group=None, device=None):
    """(smallest, largest) key over all ranks (two all-reduces of one value),
    None when every shard is empty."""
    import torch
    import torch.distributed as dist
    big = (1 << 63) - 1
    lo, hi = local if local is not None else (big, -big - 1)
    tlo = torch.tensor([lo], dtype=torch.int64, device=device)
    thi = torch.tensor([hi], dtype=torch.int64, device=device)
    dist.all_reduce(tlo, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(thi, op=dist.ReduceOp.MAX, group=group)
    lo, hi = int(tlo.item()), int(thi.item())
    return None if lo > hi else (lo, hi)


def exchange(keys, pcols, counts: Sequence[int], group=None):
    """All-to-all of the owners' runs: returns this rank's received keys and
    partial columns."""
    import torch
    import torch.distributed as dist
    dev = keys.device
    send = torch.tensor(list(counts), dtype=torch.int64, device=dev)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    rsplit = [int(x) for x in recv.tolist()]
    ssplit = [int(x) for x in counts]
    rkeys = torch.empty(sum(rsplit), dtype=keys.dtype, device=dev)
    dist.all_to_all_single(rkeys, keys, rsplit, ssplit, group=group)
    rcols = []
    for c in pcols:
        r = torch.empty(sum(rsplit), dtype=c.dtype, device=dev)
        dist.all_to_all_single(r, c, rsplit, ssplit, group=group)
        rcols.append(r)
    return rkeys, rcols


def groupby_sharded(ctx, keys, cols: Sequence = (), aggs: Sequence = (("count", None),), group=None,
                    unsigned_keys: bool = False, unsigned_cols: Sequence[bool] = (), knobs=None, ops=None) -> Result:
    """GROUP BY over the rows of all ranks of `group`; every rank calls it with
    its own shard and gets back the groups it owns, in key order."""
    import torch.distributed as dist
    ops = ops or DeviceOps(ctx)
    plan = plan_partials(aggs)
    nparts = dist.get_world_size(group)
    lk, lcols = ops.local(keys, cols, plan.partials, unsigned_keys, unsigned_cols, knobs)
    rng = global_range(key_range(lk, unsigned_keys), group, lk.device)
    counts = owner_counts(lk, range_cuts(*rng, nparts), unsigned_keys) if rng else [0] * nparts
    rk, rcols = exchange(lk, lcols, counts, group)
    fk, fa = merge_partials(ops, rk, rcols, plan, unsigned_keys)
    return Result(fk, fa, len(fk))
