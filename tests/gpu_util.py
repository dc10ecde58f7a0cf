"""Helpers shared by the GPU parity tests: run the CUDA path through the C ABI,
run the oracle on the same bytes, compare."""
import numpy as np

import cpu_oracle as O

# fp32 SUM: the oracle adds a group's values one by one in fp64.  The GPU sums
# them exactly in shared memory (128-bit fixed point) and adds partial sums
# into HBM tables with fp64 atomics, in no fixed order.  Tolerance, per group
# of n values:
#   |gpu - oracle| <= 1e-6 * |oracle| + 2 (n - 1) * 2^-53 * sum(|x|)
# The first term is the 1e-6 relative bound of the FP64 oracle.  The second is
# the worst-case rounding error of the two fp64 summations, (n - 1) u sum|x|
# each with u = 2^-53 (recursive summation; Higham, "Accuracy and Stability of
# Numerical Algorithms", 2nd ed., section 4.2).  It exceeds the first only for
# groups whose sum nearly cancels (sum|x| / |sum| above about 5e9 / n), where
# the FP64 oracle itself is not accurate to 1e-6; compare() counts them.
FP_RTOL = 1e-6
U_FP64 = 2.0 ** -53


def fp_bound(expected, absum, count):
    """Allowed |gpu - oracle| for fp32 SUMs (or AVGs, with absum and expected
    both divided by the count) of `count` values per group."""
    n1 = np.maximum(np.asarray(count, dtype=np.float64) - 1.0, 0.0)
    return FP_RTOL * np.abs(expected) + 2.0 * n1 * U_FP64 * 1.0001 * np.asarray(absum)


def to_device(a: np.ndarray):
    import torch
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def sort_result(keys: np.ndarray, aggs: list, unsigned: bool):
    k = keys.view(np.uint32) if unsigned and keys.dtype == np.int32 else keys
    order = np.argsort(k, kind="stable")
    return k[order], [a[order] for a in aggs]


def compare(gk, gaggs, keys, cols, aggs, label="", nthreads=8, presorted=False, oracle=None):
    """gk/gaggs: the CUDA result (numpy, any order unless presorted);
    keys/cols: the input.  Keys and integer aggregates must be bit-exact; fp32
    SUMs within fp_bound.  oracle: the oracle's (keys, aggs) when already
    computed.  Returns the number of fp groups that needed the second term of
    fp_bound (nearly cancelling sums)."""
    unsigned = keys.dtype == np.uint32
    if not presorted:
        gk, gaggs = sort_result(np.asarray(gk), [np.asarray(a) for a in gaggs], unsigned)
    ok, oaggs = oracle if oracle is not None else O.groupby(keys, cols, aggs, nthreads=nthreads)
    assert len(gk) == len(ok), f"{label}: {len(gk)} groups vs oracle {len(ok)}"
    np.testing.assert_array_equal(gk, ok, err_msg=f"{label}: keys")
    abs_needed = [i for i, (op, c) in enumerate(aggs) if op == "sum" and c is not None and cols[c].dtype == np.float32]
    absums, counts = {}, None
    if abs_needed:
        _, sa = O.groupby(keys, cols, [("sumabs", aggs[i][1]) for i in abs_needed] + [("count", None)],
                          nthreads=nthreads)
        absums = dict(zip(abs_needed, sa[:-1]))
        counts = sa[-1]
    cancelling = 0
    for i, (g, o) in enumerate(zip(gaggs, oaggs)):
        if i in absums:
            err = np.abs(g - o)
            bound = fp_bound(o, absums[i], counts)
            bad = np.nonzero(err > bound)[0]
            assert len(bad) == 0, f"{label}: agg {aggs[i]} fp error at {bad[:5]}: {g[bad[:5]]} vs {o[bad[:5]]}"
            cancelling += int(np.count_nonzero(err > FP_RTOL * np.abs(o)))
        else:
            np.testing.assert_array_equal(g, o, err_msg=f"{label}: agg {aggs[i]}")
    return cancelling


def run_gpu(ctx, keys, cols, aggs, knobs=None, capacity=None):
    dk = to_device(keys)
    dcols = [to_device(c) for c in cols]
    res = ctx.groupby(dk, dcols, aggs, knobs=knobs, capacity=capacity, unsigned_keys=keys.dtype == np.uint32,
                      unsigned_cols=[c.dtype == np.uint32 for c in cols])
    gk = res.keys.cpu().numpy()
    if keys.dtype == np.uint32:
        gk = gk.view(np.uint32)
    return gk, [a.cpu().numpy() for a in res.aggs], res
