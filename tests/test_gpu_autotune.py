"""gba_autotune: picks knobs by timing the caller's queries; the knobs it returns
must give correct results, and its choice is never slower than its start."""
import numpy as np
import pytest
import torch

from cpu_gpu_coprocess_groupby_agg_b200 import Context, gen_device, gen_spec, make_knobs
from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E
from gpu_util import compare

pytestmark = pytest.mark.gpu


def _queries():
    rng = np.random.default_rng(3)
    out = []
    for i in range(12):
        n = int(2 ** rng.uniform(14, 21))
        ndv = int(np.exp(rng.uniform(np.log(16), np.log(n // 2))))
        sp = gen_spec(700 + i, 64 if i % 2 else 32, ndv, float(rng.uniform(0, 1.2)), [("i64", 0, 1 << 31)])
        k, c = gen_device(sp, n)
        out.append((k, c, [("sum", 0), ("count", None)]))
    return out


@pytest.mark.parametrize("sizing", ["plain", "learned"])
def test_autotune_batch(sizing):
    ctx = Context(0)
    E.load_default(ctx)
    qs = _queries()
    outs = ctx.batch_outputs(qs)
    base = make_knobs(sizing=sizing)
    best, ms = ctx.autotune(qs, knobs=base, outs=outs, reps=2)
    assert ms > 0 and best.sizing == base.sizing
    res = ctx.groupby_batch(qs, knobs=best, outs=outs)
    for (k, c, aggs), r in zip(qs, res):
        compare(r.keys.cpu().numpy(), [a.cpu().numpy() for a in r.aggs], k.cpu().numpy(),
                [x.cpu().numpy() for x in c], aggs, "autotuned batch")
    ctx.close()


def test_autotune_single_query_searches_partition_bits():
    ctx = Context(0)
    sp = gen_spec(42, 64, 1 << 18, 0.0, [("i64", 0, 1 << 20)])
    k, c = gen_device(sp, 1 << 21)
    q = [(k, c, [("sum", 0), ("count", None)])]
    outs = ctx.batch_outputs(q)
    base = make_knobs(sizing="plain", strategy="partition")
    best, ms = ctx.autotune(q, knobs=base, outs=outs, reps=2)
    assert ms > 0
    r = ctx.groupby(k, c, q[0][2], knobs=best, out=outs[0])
    compare(r.keys.cpu().numpy(), [a.cpu().numpy() for a in r.aggs], k.cpu().numpy(), [x.cpu().numpy() for x in c],
            q[0][2], "autotuned single")
    ctx.close()
