"""Nullable value columns (Arrow validity bitmaps) and COUNT(col).

Expected values: the oracle run over the rows whose column value is present,
placed on the full set of groups (the oracle over every row); a group with no
present value gets validity 0, SUM 0, MIN the column type's largest value, MAX
its smallest, AVG NaN and COUNT(col) 0.  Integer results bit-exact, fp32 SUM
within the fp32-SUM tolerance.  Covered: both strategies, key order, integer
and fp32 columns, a column with no present value, a bitmap with every value
present, the batch entry point, and the refusals (null keys, the host-resident
entry point, a rewrite needing more than four columns)."""
import ctypes as C

import numpy as np
import pytest

import cpu_oracle as O
from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
from cpu_gpu_coprocess_groupby_agg_b200.api import build_query, parse_aggs
from gpu_util import fp_bound, sort_result, to_device

pytestmark = pytest.mark.gpu

def _data(n, ndv, seed, p_null=(0.3, 0.5, 0.2)):
    rng = np.random.default_rng(seed)
    dom = rng.integers(-(1 << 40), 1 << 40, size=ndv, dtype=np.int64)
    keys = dom[np.minimum(rng.zipf(1.3, size=n), ndv) - 1]  # a long tail of one-row groups
    cols = [rng.integers(-(1 << 40), 1 << 40, size=n, dtype=np.int64),
            rng.integers(-1000, 1000, size=n, dtype=np.int32).astype(np.int32),
            rng.standard_normal(n).astype(np.float32)]
    valid = [rng.random(n) >= p for p in p_null]
    return keys, cols, valid


def _bitmap(v):
    return np.packbits(v.astype(np.uint8), bitorder="little")


def _expected(keys, cols, valid, op, c):
    """(group keys, values, validity) of one aggregate over nullable column c."""
    gk, (cnt,) = O.groupby(keys, cols, [("count", None)], nthreads=8)
    m = valid[c]
    pk, (pc,) = O.groupby(keys[m], [x[m] for x in cols], [("count", None)], nthreads=8)
    pos = np.searchsorted(gk, pk)
    present = np.zeros(len(gk), dtype=np.uint8)
    present[pos] = 1
    if op == "count_valid":
        out = np.zeros(len(gk), dtype=np.int64)
        out[pos] = pc
        return gk, out, np.ones(len(gk), dtype=np.uint8), None
    base_op = "sum" if op == "avg" else op
    _, (pv,) = O.groupby(keys[m], [x[m] for x in cols], [(base_op, c)], nthreads=8)
    absum = None
    if pv.dtype == np.float64 or op == "avg":
        out = np.full(len(gk), np.nan if op == "avg" else 0.0)
        out[pos] = pv / pc if op == "avg" else pv
        if cols[c].dtype == np.float32:
            _, (a,) = O.groupby(keys[m], [x[m] for x in cols], [("sumabs", c)], nthreads=8)
            absum = np.zeros(len(gk))
            absum[pos] = fp_bound(out[pos], a / pc if op == "avg" else a, pc)  # the allowed error
    else:
        info = np.iinfo(cols[c].dtype)
        fill = {"sum": 0, "min": int(info.max), "max": int(info.min)}[op]
        out = np.full(len(gk), fill, dtype=np.int64)
        out[pos] = pv
    return gk, out, present, absum


def _check(res, keys, cols, valid, aggs, label, presorted=False):
    gk = res.keys.cpu().numpy()
    ga = [a.cpu().numpy() for a in res.aggs]
    gv = [v.cpu().numpy() for v in res.valid]
    if not presorted:
        order = np.argsort(gk, kind="stable")
        gk, ga, gv = gk[order], [a[order] for a in ga], [v[order] for v in gv]
    for i, (op, c) in enumerate(aggs):
        msg = f"{label}: aggregate {i} ({op} of column {c})"
        if op == "count":
            ek, (e,) = O.groupby(keys, cols, [("count", None)], nthreads=8)
            np.testing.assert_array_equal(gk, ek, err_msg=msg)
            np.testing.assert_array_equal(ga[i], e, err_msg=msg)
            assert (gv[i] == 1).all(), msg
            continue
        ek, e, ev, absum = _expected(keys, cols, valid, op, c)
        np.testing.assert_array_equal(gk, ek, err_msg=msg)
        np.testing.assert_array_equal(gv[i], ev, err_msg=msg + " validity")
        if absum is not None:
            ok = np.isclose(ga[i], e, rtol=0, atol=0, equal_nan=True) | (np.abs(ga[i] - e) <= absum)
            assert ok.all(), msg
        else:
            np.testing.assert_array_equal(ga[i], e, err_msg=msg)


# rewritten: column 0 as a zero-filled copy and a presence column, column 1 as
# a presence column and a MIN copy (four columns, the limit)
AGGS = [("sum", 0), ("count", None), ("count_valid", 1), ("min", 1), ("avg", 0)]


@pytest.mark.parametrize("strategy", ["table", "partition"])
@pytest.mark.parametrize("sort_output", [0, 1])
def test_nullable_matches_oracle(ctx, strategy, sort_output):
    keys, cols, valid = _data(300_000, 50_000, seed=3)
    res = ctx.groupby(to_device(keys), [to_device(c) for c in cols], AGGS,
                      col_valid=[to_device(_bitmap(v)) for v in valid], agg_valid=True,
                      knobs=dict(strategy=strategy, sort_output=sort_output))
    _check(res, keys, cols, valid, AGGS, f"{strategy}", presorted=bool(sort_output))


def test_nullable_fp32(ctx):
    keys, cols, valid = _data(200_000, 30_000, seed=6)
    aggs = [("sum", 2), ("avg", 2), ("count", None)]
    res = ctx.groupby(to_device(keys), [to_device(c) for c in cols], aggs,
                      col_valid=[None, None, to_device(_bitmap(valid[2]))], agg_valid=True)
    _check(res, keys, cols, valid, aggs, "fp32")


def test_nullable_all_absent_and_all_present(ctx):
    keys, cols, _ = _data(40_000, 3_000, seed=8)
    valid = [np.zeros(len(keys), bool), np.ones(len(keys), bool), np.ones(len(keys), bool)]
    aggs = [("sum", 0), ("avg", 0), ("count_valid", 0), ("sum", 1)]
    res = ctx.groupby(to_device(keys), [to_device(c) for c in cols], aggs,
                      col_valid=[to_device(_bitmap(v)) for v in valid], agg_valid=True)
    _check(res, keys, cols, valid, aggs, "all absent / all present")
    assert (res.valid[0].cpu().numpy() == 0).all() and (res.valid[3].cpu().numpy() == 1).all()


def test_nullable_without_validity_outputs(ctx):
    """SUM / MAX over a nullable column with no validity requested: no presence
    column is written; values as documented for all-absent groups."""
    keys, cols, valid = _data(100_000, 20_000, seed=5)
    aggs = [("sum", 1), ("max", 1)]
    res = ctx.groupby(to_device(keys), [to_device(c) for c in cols], aggs,
                      col_valid=[None, to_device(_bitmap(valid[1]))])
    assert res.valid is None
    gk, ga = sort_result(res.keys.cpu().numpy(), [a.cpu().numpy() for a in res.aggs], False)
    for i, (op, c) in enumerate(aggs):
        ek, e, _, _ = _expected(keys, cols, valid, op, c)
        np.testing.assert_array_equal(gk, ek)
        np.testing.assert_array_equal(ga[i], e, err_msg=op)


def test_nullable_batch(ctx):
    k1, c1, v1 = _data(80_000, 9_000, seed=1)
    rng = np.random.default_rng(2)
    k2 = rng.integers(-30, 30, size=20_000).astype(np.int64)
    c2 = [rng.integers(-9, 9, size=20_000, dtype=np.int64)]
    aggs1 = [("avg", 1), ("count_valid", 0), ("sum", 0)]
    aggs2 = [("sum", 0), ("count", None)]
    qs = [(to_device(k1), [to_device(c) for c in c1], aggs1, False, [], [to_device(_bitmap(v)) for v in v1]),
          (to_device(k2), [to_device(c) for c in c2], aggs2)]
    outs = ctx.batch_outputs(qs)
    import torch
    outs[0] = (outs[0][0], outs[0][1], [torch.empty(outs[0][0].numel(), dtype=torch.uint8, device="cuda")
                                         for _ in aggs1])
    res = ctx.groupby_batch(qs, outs=outs)
    _check(res[0], k1, c1, v1, aggs1, "batch query 0")
    gk, ga = sort_result(res[1].keys.cpu().numpy(), [a.cpu().numpy() for a in res[1].aggs], False)
    ek, eo = O.groupby(k2, c2, aggs2, nthreads=8)
    np.testing.assert_array_equal(gk, ek)
    for g, e in zip(ga, eo):
        np.testing.assert_array_equal(g, e)


def test_nullable_refusals(ctx):
    keys, cols, valid = _data(1_000, 100, seed=4)
    dk, dc = to_device(keys), [to_device(c) for c in cols]
    bm = [to_device(_bitmap(v)) for v in valid]
    # five rewritten columns: column 0 as SUM, MIN and MAX copies plus its presence column, column 1's copy
    with pytest.raises(A.GbaError) as e:
        ctx.groupby(dk, dc, [("sum", 0), ("min", 0), ("max", 0), ("sum", 1)], col_valid=bm, agg_valid=True)
    assert e.value.status == A.ERR_UNSUPPORTED
    lib = A.lib()
    kn = A.Knobs()
    lib.gba_default_knobs(C.byref(kn))
    ng = C.c_int64(0)
    # null keys
    q = build_query(len(keys), dk.data_ptr(), A.I64, [(dc[0].data_ptr(), A.I64)], parse_aggs([("sum", 0)]))
    q.key.valid = bm[0].data_ptr()
    import torch
    ok_, oa = torch.empty(1001, dtype=torch.int64, device="cuda"), torch.empty(1001, dtype=torch.int64, device="cuda")
    o = A.Output()
    o.keys, o.capacity = ok_.data_ptr(), 1001
    o.aggs[0] = oa.data_ptr()
    st = lib.gba_groupby(ctx._h, C.byref(q), C.byref(o), C.byref(kn),
                         C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(ng))
    assert st == A.ERR_UNSUPPORTED
    # the host-resident entry point takes no validity bitmap
    hb = _bitmap(valid[0])
    q = build_query(len(keys), keys.ctypes.data, A.I64, [(cols[0].ctypes.data, A.I64, hb.ctypes.data)],
                    parse_aggs([("sum", 0)]))
    hk, ha = np.empty(1001, np.int64), np.empty(1001, np.int64)
    o = A.Output()
    o.keys, o.capacity = hk.ctypes.data, 1001
    o.aggs[0] = ha.ctypes.data
    st = lib.gba_groupby_host(ctx._h, C.byref(q), C.byref(o), C.byref(kn), C.c_void_p(0), C.byref(ng))
    assert st == A.ERR_UNSUPPORTED
    torch.cuda.synchronize()


@pytest.mark.parametrize("batch", [False, True])
def test_nullable_composite_sorted_together(ctx, batch):
    """The rewrites stacked: a nullable column, a composite key, AVG and key
    order in one query (alone and through the batch entry point)."""
    import torch
    rng = np.random.default_rng(12)
    n = 60_000
    k1 = rng.integers(-40, 40, size=n).astype(np.int32)
    k2 = rng.integers(0, 50, size=n).astype(np.int32)
    v = rng.integers(-1000, 1000, size=n, dtype=np.int64)
    valid = rng.random(n) >= 0.4
    valid[(k1 == 7) & (k2 == 3)] = False  # one group with no present value
    aggs = [("avg", 0), ("count_valid", 0), ("count", None)]
    dk = (to_device(k1), to_device(k2))
    bm = [to_device(_bitmap(valid))]
    if batch:
        q = [(dk, [to_device(v)], aggs, False, [], bm)]
        outs = ctx.batch_outputs(q)
        outs[0] = (outs[0][0], outs[0][1], [torch.empty(n + 1, dtype=torch.uint8, device="cuda") for _ in aggs])
        r = ctx.groupby_batch(q, outs=outs, knobs=dict(sort_output=1))[0]
    else:
        r = ctx.groupby(dk, [to_device(v)], aggs, col_valid=bm, agg_valid=True, knobs=dict(sort_output=1))
    g1, g2 = (t.cpu().numpy() for t in r.keys)
    # expected, in (k1, k2) order: the oracle on a 64-bit key that orders like the pair
    comb = (k1.astype(np.int64) << 32) | (k2.astype(np.int64) & 0xFFFFFFFF)
    ek, (cnt,) = O.groupby(comb, [v], [("count", None)], nthreads=8)
    pk, (s, c) = O.groupby(comb[valid], [v[valid]], [("sum", 0), ("count", None)], nthreads=8)
    pos = np.searchsorted(ek, pk)
    avg = np.full(len(ek), np.nan)
    avg[pos] = s.astype(np.float64) / c
    cv = np.zeros(len(ek), dtype=np.int64)
    cv[pos] = c
    present = np.zeros(len(ek), dtype=np.uint8)
    present[pos] = 1
    np.testing.assert_array_equal(g1, (ek >> 32).astype(np.int32))
    np.testing.assert_array_equal(g2, (ek & 0xFFFFFFFF).astype(np.int32))
    np.testing.assert_array_equal(r.aggs[0].cpu().numpy(), avg)
    np.testing.assert_array_equal(r.aggs[1].cpu().numpy(), cv)
    np.testing.assert_array_equal(r.aggs[2].cpu().numpy(), cnt)
    np.testing.assert_array_equal(r.valid[0].cpu().numpy(), present)
    assert present.min() == 0  # the all-absent group is there
