"""Helpers shared by the GPU parity tests: run the CUDA path through the C ABI,
run the oracle on the same bytes, compare."""
import numpy as np

import cpu_oracle as O

# fp32 SUM accumulates in fp64 on both sides, in different orders.  Tolerance:
# |gpu - oracle| <= 1e-6 * |oracle| + 1e-12 * sum(|x|)   (relative 1e-6 of the
# FP64 oracle, with an absolute floor tied to the sum's condition number).
FP_RTOL = 1e-6
FP_ABS_PER_ABSSUM = 1e-12


def to_device(a: np.ndarray):
    import torch
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def sort_result(keys: np.ndarray, aggs: list, unsigned: bool):
    k = keys.view(np.uint32) if unsigned and keys.dtype == np.int32 else keys
    order = np.argsort(k, kind="stable")
    return k[order], [a[order] for a in aggs]


def compare(gk, gaggs, keys, cols, aggs, label=""):
    """gk/gaggs: the CUDA result (numpy, any order); keys/cols: the input."""
    unsigned = keys.dtype == np.uint32
    gk, gaggs = sort_result(np.asarray(gk), [np.asarray(a) for a in gaggs], unsigned)
    ok, oaggs = O.groupby(keys, cols, aggs, nthreads=8)
    assert len(gk) == len(ok), f"{label}: {len(gk)} groups vs oracle {len(ok)}"
    np.testing.assert_array_equal(gk, ok, err_msg=f"{label}: keys")
    abs_needed = [i for i, (op, c) in enumerate(aggs) if op == "sum" and c is not None and cols[c].dtype == np.float32]
    absums = {}
    if abs_needed:
        _, sa = O.groupby(keys, cols, [("sumabs", aggs[i][1]) for i in abs_needed], nthreads=8)
        absums = dict(zip(abs_needed, sa))
    for i, (g, o) in enumerate(zip(gaggs, oaggs)):
        if i in absums:
            err = np.abs(g - o)
            bound = FP_RTOL * np.abs(o) + FP_ABS_PER_ABSSUM * absums[i]
            bad = np.nonzero(err > bound)[0]
            assert len(bad) == 0, f"{label}: agg {aggs[i]} fp error at {bad[:5]}: {g[bad[:5]]} vs {o[bad[:5]]}"
        else:
            np.testing.assert_array_equal(g, o, err_msg=f"{label}: agg {aggs[i]}")


def run_gpu(ctx, keys, cols, aggs, knobs=None, capacity=None):
    dk = to_device(keys)
    dcols = [to_device(c) for c in cols]
    res = ctx.groupby(dk, dcols, aggs, knobs=knobs, capacity=capacity, unsigned_keys=keys.dtype == np.uint32,
                      unsigned_cols=[c.dtype == np.uint32 for c in cols])
    gk = res.keys.cpu().numpy()
    if keys.dtype == np.uint32:
        gk = gk.view(np.uint32)
    return gk, [a.cpu().numpy() for a in res.aggs], res
