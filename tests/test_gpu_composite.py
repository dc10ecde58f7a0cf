"""Composite keys: GROUP BY (key, key2) over two 32-bit key columns.

Expected results come from the oracle run on a 64-bit key built in the test by
a different bijection than the library's (first key in the high word as is,
second key's bits in the low word), decoded back into the pair and ordered
lexicographically by (key, key2) in each key's own signedness.  Keys and
integer aggregates must be bit-exact; with sort_output the library's rows must
already be in that order.  Covered: every signedness combination, both
strategies, the extreme keys, AVG, the batch entry point beside single-key
queries, and the refusals (a 64-bit second key; the host-resident entry
point)."""
import ctypes as C

import numpy as np
import pytest

import cpu_oracle as O
from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
from cpu_gpu_coprocess_groupby_agg_b200.api import build_query, parse_aggs
from gpu_util import to_device

pytestmark = pytest.mark.gpu


def _pairs(n, t1, t2, nd1, nd2, seed, extremes=False):
    rng = np.random.default_rng(seed)

    def dom(t, nd):
        info = np.iinfo(t)
        d = rng.integers(int(info.min), int(info.max) + 1, size=nd, dtype=np.int64)
        if extremes:
            d[:4] = [info.min, info.max, 0, info.max if t == np.uint32 else -1]
        return d.astype(t)

    d1, d2 = dom(t1, nd1), dom(t2, nd2)
    k1 = d1[rng.integers(0, nd1, size=n)]
    k2 = d2[rng.integers(0, nd2, size=n)]
    cols = [rng.integers(-(1 << 40), 1 << 40, size=n, dtype=np.int64), rng.integers(-100, 100, size=n, dtype=np.int32)]
    return k1, k2, cols


def _expected(k1, k2, cols, aggs):
    comb = (k1.astype(np.int64) << 32) | k2.view(np.uint32).astype(np.int64)
    ck, outs = O.groupby(comb, cols, aggs, nthreads=8)
    e1 = (ck >> 32).astype(np.int64)
    e1 = (e1 & 0xFFFFFFFF).astype(np.uint32) if k1.dtype == np.uint32 else e1.astype(np.int32)
    e2 = (ck & 0xFFFFFFFF).astype(np.uint32)
    e2 = e2 if k2.dtype == np.uint32 else e2.view(np.int32)
    order = np.lexsort((e2, e1))
    return e1[order], e2[order], [o[order] for o in outs]


def _got(r, k1, k2):
    g1, g2 = (t.cpu().numpy() for t in r.keys)
    g1 = g1.view(np.uint32) if k1.dtype == np.uint32 else g1
    g2 = g2.view(np.uint32) if k2.dtype == np.uint32 else g2
    return g1, g2, [a.cpu().numpy() for a in r.aggs]


def _check(r, k1, k2, cols, aggs, sorted_output, label):
    e1, e2, eo = _expected(k1, k2, cols, aggs)
    g1, g2, go = _got(r, k1, k2)
    assert len(g1) == len(e1), f"{label}: {len(g1)} groups vs {len(e1)}"
    if not sorted_output:
        order = np.lexsort((g2, g1))
        g1, g2, go = g1[order], g2[order], [a[order] for a in go]
    np.testing.assert_array_equal(g1, e1, err_msg=f"{label}: first keys")
    np.testing.assert_array_equal(g2, e2, err_msg=f"{label}: second keys")
    for a, (g, e) in enumerate(zip(go, eo)):
        np.testing.assert_array_equal(g, e, err_msg=f"{label}: aggregate {a}")


AGGS = [("sum", 0), ("count", None), ("min", 1), ("max", 0)]


@pytest.mark.parametrize("strategy", ["table", "partition"])
@pytest.mark.parametrize("t1,t2", [(np.int32, np.int32), (np.uint32, np.int32), (np.int32, np.uint32),
                                   (np.uint32, np.uint32)])
@pytest.mark.parametrize("sort_output", [0, 1])
def test_composite_matches_oracle(ctx, strategy, t1, t2, sort_output):
    k1, k2, cols = _pairs(250_000, t1, t2, 300, 400, seed=11, extremes=True)
    r = ctx.groupby((to_device(k1), to_device(k2)), [to_device(c) for c in cols], AGGS,
                    unsigned_keys=(t1 == np.uint32, t2 == np.uint32),
                    knobs=dict(strategy=strategy, sort_output=sort_output))
    _check(r, k1, k2, cols, AGGS, sort_output, f"{strategy} {np.dtype(t1).name},{np.dtype(t2).name}")


def test_composite_avg(ctx):
    k1, k2, cols = _pairs(80_000, np.int32, np.int32, 50, 60, seed=4)
    r = ctx.groupby((to_device(k1), to_device(k2)), [to_device(c) for c in cols], [("avg", 0)],
                    knobs=dict(sort_output=1))
    e1, e2, (s, c) = _expected(k1, k2, cols, [("sum", 0), ("count", None)])
    g1, g2, (avg,) = _got(r, k1, k2)
    np.testing.assert_array_equal(g1, e1)
    np.testing.assert_array_equal(g2, e2)
    np.testing.assert_array_equal(avg, s.astype(np.float64) / c.astype(np.float64))


def test_composite_in_batch(ctx):
    ka1, ka2, ca = _pairs(70_000, np.int32, np.uint32, 200, 300, seed=1)
    kb1, kb2, cb = _pairs(5_000, np.uint32, np.int32, 10, 10, seed=2, extremes=True)
    rng = np.random.default_rng(3)
    ks = rng.integers(-50, 50, size=30_000).astype(np.int64)
    cs = [rng.integers(-9, 9, size=30_000, dtype=np.int64)]
    aggs = [("sum", 0), ("count", None)]
    qs = [((to_device(ka1), to_device(ka2)), [to_device(c) for c in ca], aggs, (False, True)),
          (to_device(ks), [to_device(c) for c in cs], aggs),
          ((to_device(kb1), to_device(kb2)), [to_device(c) for c in cb], aggs, (True, False))]
    for sort_output in (0, 1):
        res = ctx.groupby_batch(qs, knobs=dict(sort_output=sort_output))
        _check(res[0], ka1, ka2, ca, aggs, sort_output, "batch query 0")
        _check(res[2], kb1, kb2, cb, aggs, sort_output, "batch query 2")
        ok, oo = O.groupby(ks, cs, aggs, nthreads=8)
        gk = res[1].keys.cpu().numpy()
        order = np.arange(len(gk)) if sort_output else np.argsort(gk)
        np.testing.assert_array_equal(gk[order], ok)
        for g, e in zip(res[1].aggs, oo):
            np.testing.assert_array_equal(g.cpu().numpy()[order], e)


def test_composite_refusals(ctx):
    import torch
    k1 = to_device(np.arange(100, dtype=np.int32))
    k64 = to_device(np.arange(100, dtype=np.int64))
    v = to_device(np.ones(100, dtype=np.int64))
    with pytest.raises(A.GbaError) as e:
        ctx.groupby((k1, k64), [v], [("sum", 0)])
    assert e.value.status == A.ERR_UNSUPPORTED
    # the host-resident entry point takes no composite key
    hk = np.arange(100, dtype=np.int32)
    hv = np.ones(100, dtype=np.int64)
    q = build_query(100, hk.ctypes.data, A.I32, [(hv.ctypes.data, A.I64)], parse_aggs([("sum", 0)]),
                    (hk.ctypes.data, A.I32))
    ok, oa, ok2 = np.empty(101, np.int32), np.empty(101, np.int64), np.empty(101, np.int32)
    o = A.Output()
    o.keys, o.keys2, o.capacity = ok.ctypes.data, ok2.ctypes.data, 101
    o.aggs[0] = oa.ctypes.data
    kn = A.Knobs()
    A.lib().gba_default_knobs(C.byref(kn))
    ng = C.c_int64(0)
    st = A.lib().gba_groupby_host(ctx._h, C.byref(q), C.byref(o), C.byref(kn), C.c_void_p(0), C.byref(ng))
    assert st == A.ERR_UNSUPPORTED
    torch.cuda.synchronize()
