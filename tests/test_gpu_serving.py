"""The serving loop (gba_server_*): continuous batching over CUDA streams under
a device-memory budget.

The central check: every request's result is the same alone and in the mix.
Requests of many shapes (32/64-bit keys, skewed and uniform, an fp32 SUM,
one request large enough to run alone) are submitted together to a server
with several lanes, so they run as batches on concurrent streams; each result
is compared with the same query run alone through gba_groupby on its own
context - integer aggregates bit-exact, fp32 SUMs within 1e-6 relative - and
with the oracle.
"""
import numpy as np
import pytest
import torch

import cpu_oracle as O
from cpu_gpu_coprocess_groupby_agg_b200 import Context, Server, gen_device, gen_spec, make_knobs
from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E
from gpu_util import FP_RTOL, compare

pytestmark = pytest.mark.gpu


def _requests():
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(40):
        n = int(2 ** rng.uniform(12, 20))
        ndv = int(np.exp(rng.uniform(np.log(16), np.log(max(17, n // 2)))))
        bits = 64 if i % 2 else 32
        s = float(rng.uniform(0, 1.5))
        if i % 7 == 3:
            sp = gen_spec(500 + i, bits, ndv, s, [("i64", -(1 << 31), 1 << 31), ("normal",)])
            aggs = [("sum", 0), ("count", None), ("min", 0), ("max", 0), ("sum", 1)]
        else:
            sp = gen_spec(500 + i, bits, ndv, s, [("i64", 0, 1 << 31)])
            aggs = [("sum", 0), ("count", None)]
        reqs.append((sp, n, aggs))
    # one request above batch_rows: it runs alone on a lane
    reqs.append((gen_spec(999, 64, 1 << 18, 0.0, [("i64", 0, 1 << 20)]), 3 << 20, [("sum", 0), ("count", None)]))
    return reqs


def _outputs(keys, cols, aggs):
    n = keys.numel()
    ok = torch.empty(n + 1, dtype=keys.dtype, device=keys.device)
    oa = [torch.empty(n + 1, dtype=torch.float64 if (op == "sum" and c is not None and cols[c].dtype == torch.float32)
                      else torch.int64, device=keys.device) for op, c in aggs]
    return ok, oa


def _sorted(keys, aggs, g):
    k = keys[:g].cpu().numpy()
    o = np.argsort(k, kind="stable")
    return k[o], [a[:g].cpu().numpy()[o] for a in aggs]


@pytest.mark.parametrize("sizing", ["plain", "learned"])
def test_results_same_alone_and_in_the_mix(sizing):
    reqs = _requests()
    data = [gen_device(sp, n) for sp, n, _ in reqs]
    torch.cuda.synchronize()
    params = E.load_weights() if sizing == "learned" else None
    knobs = make_knobs(sizing=sizing)
    # alone
    ctx = Context(0)
    if params is not None:
        ctx.est_load(params)
    alone = []
    for (sp, n, aggs), (k, c) in zip(reqs, data):
        r = ctx.groupby(k, c, aggs, knobs=knobs)
        alone.append(_sorted(r.keys, r.aggs, r.n_groups))
    ctx.close()
    # in the mix: everything submitted at once to 4 lanes, batches of up to 16
    sv = Server(0, lanes=4, max_batch=16, batch_rows=1 << 21, knobs=knobs, estimator_params=params)
    outs = [_outputs(k, c, aggs) for (sp, n, aggs), (k, c) in zip(reqs, data)]
    tickets = [sv.submit(k, c, aggs, o) for (sp, n, aggs), (k, c), o in zip(reqs, data, outs)]
    infos = [sv.wait(t, timeout=120) for t in tickets]
    cnt = sv.counters()
    sv.close()
    assert cnt["lane_calls"] >= 1 and cnt["batch_failures"] == 0 and cnt["lane_ms_max"] > 0, cnt
    assert max(i.batch_size for i in infos) > 1, "no request ran in a batch"
    assert len({i.lane for i in infos}) > 1, "only one lane ran"
    assert infos[-1].batch_size == 1, "the large request should run alone"
    for idx, ((sp, n, aggs), (k, c), info, (ok, oa), (ak, aa)) in enumerate(zip(reqs, data, infos, outs, alone)):
        assert info.status == A.OK, (idx, info)
        assert info.latency_ms >= info.service_ms >= 0
        mk, ma = _sorted(ok, oa, info.n_groups)
        np.testing.assert_array_equal(mk, ak, err_msg=f"request {idx}: keys")
        for j, ((op, col), x, y) in enumerate(zip(aggs, ma, aa)):
            if x.dtype == np.float64:
                np.testing.assert_allclose(x, y, rtol=FP_RTOL, atol=1e-9, err_msg=f"request {idx} agg {j}")
            else:
                np.testing.assert_array_equal(x, y, err_msg=f"request {idx} agg {j}")
    # and one of them against the oracle
    sp, n, aggs = reqs[3]
    k, c = data[3]
    compare(ok_ := outs[3][0][:infos[3].n_groups].cpu().numpy(),
            [a[:infos[3].n_groups].cpu().numpy() for a in outs[3][1]],
            k.cpu().numpy(), [x.cpu().numpy() for x in c], aggs, "oracle")


def test_budget_refuses_oversized_and_admits_within():
    sp = gen_spec(7, 64, 1000, 0.0, [("i64", 0, 100)])
    k, c = gen_device(sp, 1 << 20)
    out = _outputs(k, c, [("sum", 0)])
    sv = Server(0, lanes=2, memory_budget=8 << 20)
    with pytest.raises(A.GbaError) as e:
        sv.submit(k, c, [("sum", 0)], out)
    assert e.value.status == A.ERR_BUDGET
    sv.close()
    # a budget that fits one request at a time still finishes every request
    sv = Server(0, lanes=3, memory_budget=200 << 20)
    outs = [_outputs(k, c, [("sum", 0)]) for _ in range(6)]
    ts = [sv.submit(k, c, [("sum", 0)], o) for o in outs]
    infos = [sv.wait(t) for t in ts]
    cnt = sv.counters()
    sv.close()
    assert cnt["lane_calls"] >= 2 and cnt["ws_releases"] >= 0 and cnt["release_ms_max"] >= 0, cnt
    assert all(i.status == A.OK and i.n_groups == infos[0].n_groups for i in infos)
    assert infos[0].n_groups == len(np.unique(k.cpu().numpy()))


def test_next_done_collects_every_request():
    sp = gen_spec(8, 32, 5000, 0.8, [("i64", 0, 100)])
    k, c = gen_device(sp, 200_000)
    sv = Server(0, lanes=2, max_batch=4)
    outs = [_outputs(k, c, [("count", None)]) for _ in range(10)]
    ts = {sv.submit(k, c, [("count", None)], o) for o in outs}
    got = set()
    while len(got) < len(ts):
        info = sv.next_done(timeout=60)
        assert info is not None
        assert info.status == A.OK
        got.add(info.ticket)
    assert got == ts
    assert sv.next_done(timeout=0.01) is None
    assert sv.pending() == (0, 0, 0)
    sv.close()
