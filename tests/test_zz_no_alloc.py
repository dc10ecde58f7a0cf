"""gba_groupby_noalloc (fixed static scratch, no device allocation) through the
C ABI: the same groups and aggregates as gba_groupby and as the CPU oracle on
two calls in a row, in this process after the other tests and in a fresh
process of its own."""
import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import cpu_oracle as O

from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
from cpu_gpu_coprocess_groupby_agg_b200.api import build_query, parse_aggs

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
SCRATCH_BYTES = 16 << 20
AGGS = [("sum", 0), ("count", None), ("min", 0), ("max", 0), ("sum", 1)]


def _data(n, kdt, ndv, seed):
    rng = np.random.default_rng(seed)
    ranks = np.minimum(rng.zipf(1.2, size=n), ndv) - 1
    info = np.iinfo(kdt)
    dom = rng.integers(int(info.min), int(info.max) + 1, size=ndv, dtype=np.int64).astype(kdt)
    keys = dom[ranks]
    cols = [rng.integers(-(1 << 40), 1 << 40, size=n, dtype=np.int64), rng.standard_normal(n).astype(np.float32)]
    return keys, cols


def _noalloc(ctx, dk, dcols, aggs, unsigned_keys=False, valid_out=False):
    """Calls gba_groupby_noalloc directly through ctypes; returns (status, keys, aggs).
    valid_out: also pass a per-aggregate validity output (not supported)."""
    import torch
    n = dk.numel()
    kt = A.U32 if unsigned_keys else {torch.int32: A.I32, torch.int64: A.I64}[dk.dtype]
    ct = [{torch.int64: A.I64, torch.float32: A.F32, torch.int32: A.I32}[c.dtype] for c in dcols]
    ap = parse_aggs(aggs)
    q = build_query(n, dk.data_ptr(), kt, [(c.data_ptr(), t) for c, t in zip(dcols, ct)], ap)
    cap = max(n, 1)
    okeys = torch.empty(cap, dtype=dk.dtype, device=dk.device)
    oaggs = [torch.empty(cap, dtype=torch.float64 if (op == A.SUM and ct[col] == A.F32) else torch.int64,
                         device=dk.device) for op, col in ap]
    o = A.Output()
    o.keys = okeys.data_ptr()
    for i, t in enumerate(oaggs):
        o.aggs[i] = t.data_ptr()
    o.capacity = cap
    if valid_out:
        vbuf = torch.empty(cap, dtype=torch.uint8, device=dk.device)
        o.agg_valid[0] = vbuf.data_ptr()
    ng = C.c_int64(-1)
    s = torch.cuda.current_stream(dk.device)
    st = ctx._lib.gba_groupby_noalloc(ctx._h, C.byref(q), C.byref(o), C.c_void_p(s.cuda_stream), C.byref(ng))
    if st != A.OK:
        return st, None, None
    g = ng.value
    return st, okeys[:g].cpu().numpy(), [t[:g].cpu().numpy() for t in oaggs]


def _sorted(keys, aggs, unsigned):
    k = keys.view(np.uint32) if unsigned else keys
    order = np.argsort(k, kind="stable")
    return k[order], [a[order] for a in aggs]


def _check_same(ctx, keys, cols, aggs):
    """noalloc twice in a row == gba_groupby and == the oracle (integers
    bit-exact, fp32 sums within 1e-6 relative of the FP64 oracle)."""
    import torch
    unsigned = keys.dtype == np.uint32
    dk = torch.from_numpy(keys.view(np.int32) if unsigned else keys).cuda()
    dcols = [torch.from_numpy(c).cuda() for c in cols]
    ref = ctx.groupby(dk, dcols, aggs, unsigned_keys=unsigned)
    rk = ref.keys.cpu().numpy()
    rk, ra = _sorted(rk, [a.cpu().numpy() for a in ref.aggs], unsigned)
    ok, oa = O.groupby(keys, cols, aggs, nthreads=8)
    for call in range(2):
        st, k, a = _noalloc(ctx, dk, dcols, aggs, unsigned_keys=unsigned)
        assert st == A.OK, (call, st, ctx._lib.gba_last_error(ctx._h))
        k, a = _sorted(k, a, unsigned)
        np.testing.assert_array_equal(k, rk, err_msg=f"call {call}: keys")
        for i, (x, y) in enumerate(zip(a, ra)):
            if x.dtype == np.float64:
                np.testing.assert_allclose(x, y, rtol=1e-6, atol=0, err_msg=f"call {call}: agg {aggs[i]}")
            else:
                np.testing.assert_array_equal(x, y, err_msg=f"call {call}: agg {aggs[i]}")
        np.testing.assert_array_equal(k, ok, err_msg=f"call {call}: keys vs oracle")
        for i, (x, y) in enumerate(zip(a, oa)):
            if x.dtype == np.float64:
                np.testing.assert_allclose(x, y, rtol=1e-6, atol=0, err_msg=f"call {call}: agg {aggs[i]} vs oracle")
            else:
                np.testing.assert_array_equal(x, y, err_msg=f"call {call}: agg {aggs[i]} vs oracle")


# 5 aggregates: at most 174,727 rows fit the 16 MiB scratch
@pytest.mark.parametrize("n,kdt,ndv", [(170_003, np.int64, 5000), (100_000, np.uint32, 1024), (0, np.int64, 1),
                                       (1, np.int32, 1), (174_727, np.int32, 80_000)])
def test_noalloc_matches_groupby_twice(ctx, n, kdt, ndv):
    keys, cols = _data(n, kdt, ndv, seed=n + ndv)
    _check_same(ctx, keys, cols, AGGS)


def test_noalloc_leaves_free_device_memory_unchanged(ctx):
    import torch
    keys, cols = _data(150_000, np.int64, 3000, seed=7)
    dk = torch.from_numpy(keys).cuda()
    dcols = [torch.from_numpy(c).cuda() for c in cols]
    assert _noalloc(ctx, dk, dcols, AGGS)[0] == A.OK  # the first call may load device code
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert _noalloc(ctx, dk, dcols, AGGS)[0] == A.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_queries_beyond_the_scratch(ctx):
    import torch
    n = 400_000  # (2n + 65) * 6 words * 8 bytes > 16 MiB with 5 aggregates
    dk = torch.zeros(n, dtype=torch.int64, device="cuda")
    dcols = [torch.zeros(n, dtype=torch.int64, device="cuda"), torch.zeros(n, dtype=torch.float32, device="cuda")]
    st, _, _ = _noalloc(ctx, dk, dcols, AGGS)
    assert st == A.ERR_INVALID_ARG
    msg = ctx._lib.gba_last_error(ctx._h).decode()
    assert str(SCRATCH_BYTES) in msg and "rows" in msg, msg


def test_noalloc_refuses_a_capturing_stream(ctx):
    """The call synchronises its stream, so under stream capture it returns
    GBA_ERR_INVALID_ARG before any CUDA work (the capture stays valid)."""
    import torch
    keys, cols = _data(1000, np.int64, 50, seed=5)
    dk = torch.from_numpy(keys).cuda()
    dcols = [torch.from_numpy(c).cuda() for c in cols]
    assert _noalloc(ctx, dk, dcols, AGGS)[0] == A.OK  # address lookup outside any capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        st = _noalloc(ctx, dk, dcols, AGGS)[0]
    assert st == A.ERR_INVALID_ARG
    assert "captured" in ctx._lib.gba_last_error(ctx._h).decode()
    del g
    assert _noalloc(ctx, dk, dcols, AGGS)[0] == A.OK


def test_noalloc_rejects_validity_outputs(ctx):
    import torch
    keys, cols = _data(1000, np.int64, 50, seed=3)
    dk = torch.from_numpy(keys).cuda()
    dcols = [torch.from_numpy(c).cuda() for c in cols]
    st, _, _ = _noalloc(ctx, dk, dcols, AGGS, valid_out=True)
    assert st == A.ERR_UNSUPPORTED
    assert "agg_valid" in ctx._lib.gba_last_error(ctx._h).decode()


_FRESH = r"""
import sys
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
sys.path.insert(0, {oracle!r})
import numpy as np
from cpu_gpu_coprocess_groupby_agg_b200 import Context
import test_zz_no_alloc as T
ctx = Context(0)
keys, cols = T._data(170_000, np.int64, 20_000, seed=11)
# the no-allocation entry point runs first in this process
import torch
dk = torch.from_numpy(keys).cuda()
dcols = [torch.from_numpy(c).cuda() for c in cols]
st, k, a = T._noalloc(ctx, dk, dcols, T.AGGS)
assert st == 0, st
T._check_same(ctx, keys, cols, T.AGGS)
print("FRESH-OK")
"""


def test_noalloc_in_a_fresh_process():
    code = _FRESH.format(root=str(ROOT), tests=str(ROOT / "tests"), oracle=str(ROOT / "oracle"))
    env = dict(os.environ)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env,
                       cwd=str(ROOT))
    assert r.returncode == 0 and "FRESH-OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
