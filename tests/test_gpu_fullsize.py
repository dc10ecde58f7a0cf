"""Parity at the benchmark's full sizes, through properties that do not need
the CPU oracle to finish (it would take minutes at these sizes):

* COUNT over all groups equals the row count; SUM over all groups equals the
  column's total (int64, wrapping); fp32 SUMs add up to the column's fp64
  total within 1e-6 relative;
* keys are distinct and their number equals torch.unique's count;
* MIN <= MAX for every group;
* learned and plain sizing (different tables, different strategies) return
  the same groups with the same aggregates, bit for bit on integers.
"""
import numpy as np
import pytest
import torch

from cpu_gpu_coprocess_groupby_agg_b200 import Context, gen_device, make_knobs, workloads as W
from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E

pytestmark = pytest.mark.gpu


def _sorted(res):
    order = torch.argsort(res.keys)
    return res.keys[order], [a[order] for a in res.aggs]


def _wrap64(x: torch.Tensor) -> int:
    return int(x.sum().item()) & ((1 << 64) - 1)


def _check_properties(w, keys, cols, res):
    n = w.n
    k, aggs = _sorted(res)
    assert res.n_groups == torch.unique(keys).numel()
    assert bool((k[1:] != k[:-1]).all()), "duplicate keys"
    for (op, c), a in zip(w.aggs, aggs):
        if op == "count":
            assert int(a.sum().item()) == n
        elif op == "sum" and cols[c].dtype == torch.float32:
            tot = cols[c].double().sum().item()
            absum = cols[c].double().abs().sum().item()
            assert abs(a.sum().item() - tot) <= 1e-6 * absum
        elif op == "sum":
            assert _wrap64(a) == _wrap64(cols[c].long())
    ops = [op for op, _ in w.aggs]
    if "min" in ops and "max" in ops:
        assert bool((aggs[ops.index("min")] <= aggs[ops.index("max")]).all())
    return k, aggs


@pytest.mark.parametrize("name", ["skewed", "highcard"])
def test_single_query_full_size(name):
    w = {"skewed": W.skewed, "highcard": W.high_card}[name]()
    ctx = Context(0)
    E.load_default(ctx)
    keys, cols = gen_device(w.spec, w.n)
    got = {}
    for sizing in ("learned", "plain"):
        res = ctx.groupby(keys, cols, w.aggs, knobs=make_knobs(sizing=sizing))
        got[sizing] = _check_properties(w, keys, cols, res)
        del res
    kl, al = got["learned"]
    kp, ap = got["plain"]
    assert torch.equal(kl, kp)
    for (op, c), x, y in zip(w.aggs, al, ap):
        if x.dtype == torch.float64:
            assert torch.allclose(x, y, rtol=1e-6, atol=1e-9)
        else:
            assert torch.equal(x, y)
    ctx.close()


def test_batch_full_size():
    allq = W.batch_queries()
    ctx = Context(0)
    E.load_default(ctx)
    dq = [(*gen_device(q.spec, q.n), q.aggs) for q in allq]
    outs = ctx.batch_outputs(dq)
    res_l = ctx.groupby_batch(dq, knobs=make_knobs(sizing="learned"), outs=outs)
    sl = [_check_properties(q, k, c, r) for q, (k, c, _), r in zip(allq, dq, res_l)]
    sl = [(k.clone(), [a.clone() for a in aggs]) for k, aggs in sl]
    res_p = ctx.groupby_batch(dq, knobs=make_knobs(sizing="plain"), outs=outs)
    for q, (k, c, _), r, (kl, al) in zip(allq, dq, res_p, sl):
        kp, ap = _check_properties(q, k, c, r)
        assert torch.equal(kl, kp), q.name
        for x, y in zip(al, ap):
            assert torch.equal(x, y), q.name
    ctx.close()
