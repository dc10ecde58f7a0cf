"""Python host API over the C ABI (``include/gba.h``).

``Context.groupby`` takes device-resident torch tensors; ``Context.groupby_host``
takes numpy arrays in host memory (pinned or not) and returns numpy results.
Every call goes through ``libgba.so``; there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _abi as A

_OPS = {"sum": A.SUM, "count": A.COUNT, "min": A.MIN, "max": A.MAX, "avg": A.AVG, "count_valid": A.COUNT_VALID}


def _np_type(a: np.ndarray) -> int:
    return {np.dtype(np.int32): A.I32, np.dtype(np.uint32): A.U32, np.dtype(np.int64): A.I64,
            np.dtype(np.float32): A.F32, np.dtype(np.float64): A.F64}[a.dtype]


def _torch_type(t, unsigned: bool = False) -> int:
    import torch
    m = {torch.int32: A.U32 if unsigned else A.I32, torch.int64: A.I64, torch.float32: A.F32, torch.float64: A.F64}
    if t.dtype not in m:
        raise TypeError(f"unsupported column dtype {t.dtype}")
    return m[t.dtype]


def parse_aggs(aggs: Sequence) -> list[tuple[int, int]]:
    """[("sum", 0), ("count", None), ...] -> [(op, col), ...]"""
    out = []
    for op, col in aggs:
        o = _OPS[op] if isinstance(op, str) else int(op)
        out.append((o, 0 if col is None else int(col)))
    return out


def agg_is_fp(op: int, col_type: int) -> bool:
    """Does the aggregate's output column hold doubles (else int64)?"""
    return op == A.AVG or (op == A.SUM and col_type in (A.F32, A.F64))


def make_knobs(**kw) -> A.Knobs:
    k = A.Knobs()
    A.lib().gba_default_knobs(C.byref(k))
    for name, val in kw.items():
        if name == "sizing" and isinstance(val, str):
            val = {"plain": A.SIZING_PLAIN, "learned": A.SIZING_LEARNED, "fixed": A.SIZING_FIXED,
                   "grow": A.SIZING_GROW}[val]
        if name == "strategy" and isinstance(val, str):
            val = {"auto": A.STRATEGY_AUTO, "table": A.STRATEGY_TABLE, "partition": A.STRATEGY_PARTITION}[val]
        setattr(k, name, val)
    return k


def _split_keys(keys, unsigned_keys):
    """(first key, second key or None, unsigned flags of both): keys is a tensor
    or, for a composite key, a pair of 32-bit tensors."""
    if isinstance(keys, (tuple, list)):
        k1, k2 = keys
        u = tuple(unsigned_keys) if isinstance(unsigned_keys, (tuple, list)) else (bool(unsigned_keys),) * 2
        return k1, k2, u
    return keys, None, (bool(unsigned_keys), False)


def _empty_like_keys(keys, cap):
    import torch
    if isinstance(keys, (tuple, list)):
        return tuple(torch.empty(cap, dtype=k.dtype, device=k.device) for k in keys)
    return torch.empty(cap, dtype=keys.dtype, device=keys.device)


def _set_out_keys(o: A.Output, okeys) -> int:
    """Points o at the output key column(s); returns the capacity."""
    if isinstance(okeys, (tuple, list)):
        o.keys, o.keys2 = okeys[0].data_ptr(), okeys[1].data_ptr()
        return min(okeys[0].numel(), okeys[1].numel())
    o.keys = okeys.data_ptr()
    return okeys.numel()


def _head(okeys, g):
    return tuple(k[:g] for k in okeys) if isinstance(okeys, (tuple, list)) else okeys[:g]


def build_query(n: int, key_ptr: int, key_type: int, cols: Sequence[tuple[int, int]],
                aggs: Sequence[tuple[int, int]], key2: tuple[int, int] | None = None) -> A.Query:
    q = A.Query()
    q.n_rows = n
    q.key.type = key_type
    q.key.data = key_ptr
    if key2 is not None:
        q.key2.data, q.key2.type = key2
    q.n_cols = len(cols)
    for i, spec in enumerate(cols):  # (data pointer, type[, validity bitmap pointer])
        q.cols[i].data, q.cols[i].type = spec[0], spec[1]
        if len(spec) > 2 and spec[2]:
            q.cols[i].valid = spec[2]
    q.n_aggs = len(aggs)
    for i, (op, col) in enumerate(aggs):
        q.aggs[i].op = op
        q.aggs[i].col = col
    return q


@dataclass
class PreparedBatch:
    queries: Sequence
    outs: list
    qarr: object
    oarr: object
    ng: object


@dataclass
class Result:
    keys: object
    aggs: list
    n_groups: int
    stats: dict = field(default_factory=dict)
    valid: list | None = None  # per aggregate, uint8 per group (when requested)


class Context:
    """One device context (workspace, streams, estimator weights)."""

    def __init__(self, device: int = 0):
        self._lib = A.lib()
        h = C.c_void_p()
        A.check(self._lib.gba_create(C.byref(h), device))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gba_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self) -> dict:
        s = A.Stats()
        A.check(self._lib.gba_last_stats(self._h, C.byref(s)), self._h)
        d = {name: getattr(s, name) for name, _ in A.Stats._fields_}
        d["kernel_ms"] = list(s.kernel_ms)
        return d

    # ---- device-resident ---------------------------------------------------
    def groupby(self, keys, cols: Sequence = (), aggs: Sequence = (("count", None),), knobs=None,
                capacity: int | None = None, unsigned_keys: bool = False, stream=None, out=None,
                unsigned_cols: Sequence[bool] = (), col_valid: Sequence = (), agg_valid: bool = False) -> Result:
        """torch has no general uint32 dtype: pass uint32 data as int32 tensors
        and mark them with unsigned_keys / unsigned_cols[i].  A composite key is
        a pair of 32-bit tensors (unsigned_keys may then be a pair of flags);
        the result's keys are then a pair too.  col_valid[i]: a uint8 device
        tensor holding column i's validity bitmap (Arrow layout), or None;
        agg_valid: also return one validity byte per group and aggregate."""
        import torch
        k1, k2, uk = _split_keys(keys, unsigned_keys)
        if not k1.is_cuda:
            raise ValueError("groupby() takes device tensors; use groupby_host() for host arrays")
        n = k1.numel()
        aggs_p = parse_aggs(aggs)
        uc = list(unsigned_cols) + [False] * (len(cols) - len(unsigned_cols))
        cv = list(col_valid) + [None] * (len(cols) - len(col_valid))
        col_specs = [(c.data_ptr(), _torch_type(c, u), 0 if v is None else v.data_ptr())
                     for c, u, v in zip(cols, uc, cv)]
        q = build_query(n, k1.data_ptr(), _torch_type(k1, uk[0]), col_specs, aggs_p,
                        None if k2 is None else (k2.data_ptr(), _torch_type(k2, uk[1])))
        if out is None:
            cap = capacity if capacity is not None else max(n, 1) + 1
            okeys = _empty_like_keys(keys, cap)
            oaggs = [torch.empty(cap, dtype=torch.float64 if agg_is_fp(op, col_specs[col][1] if op != A.COUNT else 0)
                                 else torch.int64, device=k1.device) for op, col in aggs_p]
        else:
            okeys, oaggs = out
        o = A.Output()
        cap = _set_out_keys(o, okeys)
        for i, t in enumerate(oaggs):
            o.aggs[i] = t.data_ptr()
        o.capacity = cap
        ovalid = None
        if agg_valid:
            ovalid = [torch.empty(cap, dtype=torch.uint8, device=k1.device) for _ in aggs_p]
            for i, t in enumerate(ovalid):
                o.agg_valid[i] = t.data_ptr()
        kn = knobs if isinstance(knobs, A.Knobs) else make_knobs(**(knobs or {}))
        ng = C.c_int64(0)
        s = stream if stream is not None else torch.cuda.current_stream(k1.device)
        st = self._lib.gba_groupby(self._h, C.byref(q), C.byref(o), C.byref(kn), C.c_void_p(s.cuda_stream),
                                   C.byref(ng))
        A.check(st, self._h)
        g = ng.value
        return Result(_head(okeys, g), [t[:g] for t in oaggs], g, self.stats(),
                      None if ovalid is None else [t[:g] for t in ovalid])

    def batch_outputs(self, queries: Sequence, capacity: Sequence[int] | None = None) -> list:
        """Device output buffers (keys, aggs) for each query of a batch; reusable
        across calls with the same shapes."""
        import torch
        outs = []
        for i, q in enumerate(queries):
            keys, cols, aggs = q[0], q[1], q[2]
            aggs_p = parse_aggs(aggs)
            uc = list(q[4]) if len(q) > 4 else []
            uc += [False] * (len(cols) - len(uc))
            ctypes_ = [_torch_type(c, u) for c, u in zip(cols, uc)]
            k1 = _split_keys(keys, False)[0]
            cap = capacity[i] if capacity is not None else max(k1.numel(), 1) + 1
            okeys = _empty_like_keys(keys, cap)
            oaggs = [torch.empty(cap, dtype=torch.float64 if agg_is_fp(op, ctypes_[col] if op != A.COUNT else 0)
                                 else torch.int64, device=k1.device) for op, col in aggs_p]
            outs.append((okeys, oaggs))
        return outs

    def _batch_arrays(self, queries: Sequence, outs):
        nq = len(queries)
        qarr = (A.Query * max(nq, 1))()
        oarr = (A.Output * max(nq, 1))()
        for i, q in enumerate(queries):
            keys, cols, aggs = q[0], q[1], q[2]
            k1, k2, uk = _split_keys(keys, q[3] if len(q) > 3 else False)
            uc = list(q[4]) if len(q) > 4 else []
            uc += [False] * (len(cols) - len(uc))
            if not k1.is_cuda:
                raise ValueError("device tensors expected")
            cv = list(q[5]) if len(q) > 5 else []
            cv += [None] * (len(cols) - len(cv))
            col_specs = [(c.data_ptr(), _torch_type(c, u), 0 if v is None else v.data_ptr())
                         for c, u, v in zip(cols, uc, cv)]
            qarr[i] = build_query(k1.numel(), k1.data_ptr(), _torch_type(k1, uk[0]), col_specs, parse_aggs(aggs),
                                  None if k2 is None else (k2.data_ptr(), _torch_type(k2, uk[1])))
            okeys, oaggs = outs[i][0], outs[i][1]
            for a, t in enumerate(oaggs):
                oarr[i].aggs[a] = t.data_ptr()
            if len(outs[i]) > 2 and outs[i][2] is not None:  # validity bytes per aggregate
                for a, t in enumerate(outs[i][2]):
                    oarr[i].agg_valid[a] = t.data_ptr()
            oarr[i].capacity = _set_out_keys(oarr[i], okeys)
        return qarr, oarr

    def prepare_batch(self, queries: Sequence, outs=None) -> "PreparedBatch":
        """Packs a batch's query and output descriptors once, for repeated
        run_batch calls on the same tensors (the per-call Python packing of
        hundreds of descriptors otherwise costs milliseconds of host time)."""
        if outs is None:
            outs = self.batch_outputs(queries)
        qarr, oarr = self._batch_arrays(queries, outs)
        return PreparedBatch(queries, outs, qarr, oarr, (C.c_int64 * max(len(queries), 1))())

    def run_batch(self, pb: "PreparedBatch", knobs=None, stream=None) -> np.ndarray:
        """gba_groupby_batch on a prepared batch; returns the group counts
        (numpy int64, one per query).  Query i's groups are
        pb.outs[i][0][:n], [a[:n] for a in pb.outs[i][1]]."""
        import torch
        kn = knobs if isinstance(knobs, A.Knobs) else make_knobs(**(knobs or {}))
        s = stream if stream is not None else torch.cuda.current_stream(_split_keys(pb.queries[0][0], False)[0].device)
        A.check(self._lib.gba_groupby_batch(self._h, len(pb.queries), pb.qarr, pb.oarr, C.byref(kn),
                                            C.c_void_p(s.cuda_stream), pb.ng), self._h)
        return np.ctypeslib.as_array(pb.ng)[:len(pb.queries)].copy()

    def autotune(self, queries: Sequence, knobs=None, outs=None, stream=None, reps: int = 2):
        """gba_autotune over device queries (one query: gba_groupby knobs; several:
        gba_groupby_batch knobs).  Returns (best knobs, best ms per call)."""
        import torch
        if outs is None:
            outs = self.batch_outputs(queries)
        qarr, oarr = self._batch_arrays(queries, outs)
        kn = knobs if isinstance(knobs, A.Knobs) else make_knobs(**(knobs or {}))
        best = A.Knobs()
        ms = C.c_double(0)
        s = stream if stream is not None else torch.cuda.current_stream(_split_keys(queries[0][0], False)[0].device)
        A.check(self._lib.gba_autotune(self._h, len(queries), qarr, oarr, C.byref(kn), C.c_void_p(s.cuda_stream),
                                       reps, C.byref(best), C.byref(ms)), self._h)
        return best, ms.value

    def groupby_batch(self, queries: Sequence, knobs=None, stream=None, outs=None) -> list:
        """Many independent queries in one call (gba_groupby_batch).

        queries: sequence of (keys, cols, aggs[, unsigned_keys[, unsigned_cols[,
        col_valid]]]) with device tensors (keys: a tensor, or a pair of 32-bit
        tensors for a composite key; col_valid: validity bitmaps or None per
        column); outs: batch_outputs() buffers (allocated when None), each
        (keys, aggs[, validity bytes per aggregate]).
        Returns one Result per query (views into the output buffers)."""
        import torch
        nq = len(queries)
        if outs is None:
            outs = self.batch_outputs(queries)
        qarr, oarr = self._batch_arrays(queries, outs)
        kn = knobs if isinstance(knobs, A.Knobs) else make_knobs(**(knobs or {}))
        ng = (C.c_int64 * max(nq, 1))()
        dev = _split_keys(queries[0][0], False)[0].device if nq else torch.device("cuda", 0)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        A.check(self._lib.gba_groupby_batch(self._h, nq, qarr, oarr, C.byref(kn), C.c_void_p(s.cuda_stream), ng),
                self._h)
        st = self.stats()
        res = []
        for i in range(nq):
            g = ng[i]
            okeys, oaggs = outs[i][0], outs[i][1]
            ov = outs[i][2] if len(outs[i]) > 2 else None
            res.append(Result(_head(okeys, g), [t[:g] for t in oaggs], g, st,
                              None if ov is None else [t[:g] for t in ov]))
        return res

    def groupby_batch_host(self, queries: Sequence, outs: Sequence, knobs=None, stream=None) -> list:
        """gba_groupby_batch_host: many queries over HOST columns into HOST
        output buffers (pinned memory gives full link speed).

        queries: sequence of (keys, cols, aggs) with numpy arrays or CPU
        tensors; outs: per query (keys, [aggregate columns]) host buffers of
        equal capacity.  Returns one Result per query (views into outs)."""
        import torch
        nq = len(queries)
        qarr = (A.Query * max(nq, 1))()
        oarr = (A.Output * max(nq, 1))()

        def ptr_type(x):
            if isinstance(x, torch.Tensor):
                assert not x.is_cuda and x.is_contiguous(), "contiguous host tensors expected"
                return x.data_ptr(), _torch_type(x, False), x.numel()
            assert isinstance(x, np.ndarray) and x.flags.c_contiguous, "contiguous numpy arrays expected"
            return x.ctypes.data, _np_type(x), x.shape[0]

        for i, (keys, cols, aggs) in enumerate(queries):
            kp, kt, n = ptr_type(keys)
            col_specs = [ptr_type(c)[:2] for c in cols]
            qarr[i] = build_query(n, kp, kt, col_specs, parse_aggs(aggs))
            okeys, oaggs = outs[i][0], outs[i][1]
            okp, _, cap = ptr_type(okeys)
            oarr[i].keys = okp
            for a, t in enumerate(oaggs):
                oarr[i].aggs[a] = ptr_type(t)[0]
            oarr[i].capacity = cap
        kn = knobs if isinstance(knobs, A.Knobs) else make_knobs(**(knobs or {}))
        ng = (C.c_int64 * max(nq, 1))()
        s = stream if stream is not None else torch.cuda.current_stream()
        A.check(self._lib.gba_groupby_batch_host(self._h, nq, qarr, oarr, C.byref(kn), C.c_void_p(s.cuda_stream), ng),
                self._h)
        st = self.stats()
        return [Result(outs[i][0][:ng[i]], [t[:ng[i]] for t in outs[i][1]], ng[i], st) for i in range(nq)]

    # ---- learned cardinality estimator ---------------------------------------
    def est_param_count(self) -> int:
        return int(self._lib.gba_estimator_param_count())

    def est_load(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.shape == (self.est_param_count(),)
        A.check(self._lib.gba_estimator_load(self._h, p.ctypes.data_as(C.POINTER(C.c_float))), self._h)

    def est_get(self) -> np.ndarray:
        p = np.empty(self.est_param_count(), dtype=np.float32)
        A.check(self._lib.gba_estimator_get(self._h, p.ctypes.data_as(C.POINTER(C.c_float))), self._h)
        return p

    def est_predict(self, feats: np.ndarray) -> np.ndarray:
        """log2(groups) predicted for each feature row."""
        X = np.ascontiguousarray(feats, dtype=np.float32).reshape(-1, A.GBA_EST_FEATURES)
        out = np.empty(X.shape[0], dtype=np.float32)
        A.check(self._lib.gba_estimator_predict(self._h, X.shape[0], X.ctypes.data_as(C.POINTER(C.c_float)),
                                                out.ctypes.data_as(C.POINTER(C.c_float))), self._h)
        return out

    def est_features(self, keys, unsigned: bool = False, tile_rows: int = 0, stream=None) -> np.ndarray:
        """The 32 estimator features of a device key column."""
        import torch
        q = build_query(keys.numel(), keys.data_ptr(), _torch_type(keys, unsigned), [], [(A.COUNT, 0)])
        out = np.empty(A.GBA_EST_FEATURES, dtype=np.float32)
        s = stream if stream is not None else torch.cuda.current_stream(keys.device)
        A.check(self._lib.gba_estimator_features(self._h, C.byref(q), tile_rows, C.c_void_p(s.cuda_stream),
                                                 out.ctypes.data_as(C.POINTER(C.c_float))), self._h)
        return out

    def est_train(self, X: np.ndarray, log2_groups: np.ndarray, epochs: int = 100, batch: int = 128,
                  lr: float = 1e-3, seed: int = 0) -> float:
        """Trains the loaded weights on the GPU; returns the final MSE in (log2)^2."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(log2_groups, dtype=np.float32)
        loss = C.c_float(0)
        A.check(self._lib.gba_estimator_train(self._h, X.shape[0], X.ctypes.data_as(C.POINTER(C.c_float)),
                                              y.ctypes.data_as(C.POINTER(C.c_float)), epochs, batch, lr, seed,
                                              C.byref(loss)), self._h)
        return float(loss.value)

    def est_grad(self, X: np.ndarray, log2_groups: np.ndarray):
        """One forward/backward pass on the GPU: (gradients, loss) with the
        target scaled as t = log2(groups) / 32."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(log2_groups, dtype=np.float32)
        g = np.empty(self.est_param_count(), dtype=np.float32)
        loss = C.c_float(0)
        A.check(self._lib.gba_estimator_grad(self._h, X.shape[0], X.ctypes.data_as(C.POINTER(C.c_float)),
                                             y.ctypes.data_as(C.POINTER(C.c_float)),
                                             g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)), self._h)
        return g, float(loss.value)

    # ---- host-resident -----------------------------------------------------
    def groupby_host(self, keys: np.ndarray, cols: Sequence[np.ndarray] = (), aggs: Sequence = (("count", None),),
                     knobs=None, capacity: int | None = None, stream=None, out=None) -> Result:
        n = keys.shape[0]
        aggs_p = parse_aggs(aggs)
        keys = np.ascontiguousarray(keys)
        cols = [np.ascontiguousarray(c) for c in cols]
        col_specs = [(c.ctypes.data, _np_type(c)) for c in cols]
        q = build_query(n, keys.ctypes.data, _np_type(keys), col_specs, aggs_p)
        if out is None:
            cap = capacity if capacity is not None else max(n, 1) + 1
            okeys = np.empty(cap, dtype=keys.dtype)
            oaggs = [np.empty(cap, dtype=np.float64 if (op != A.COUNT and agg_is_fp(op, col_specs[col][1]))
                              else np.int64) for op, col in aggs_p]
        else:
            okeys, oaggs = out
            cap = okeys.shape[0]
        o = A.Output()
        o.keys = okeys.ctypes.data
        for i, t in enumerate(oaggs):
            o.aggs[i] = t.ctypes.data
        o.capacity = cap
        kn = knobs if isinstance(knobs, A.Knobs) else make_knobs(**(knobs or {}))
        ng = C.c_int64(0)
        sp = 0 if stream is None else stream.cuda_stream
        A.check(self._lib.gba_groupby_host(self._h, C.byref(q), C.byref(o), C.byref(kn), C.c_void_p(sp),
                                           C.byref(ng)), self._h)
        g = ng.value
        return Result(okeys[:g], [t[:g] for t in oaggs], g, self.stats())


# ---- seeded synthetic data -------------------------------------------------------
def gen_spec(seed: int, key_bits: int, ndv: int, zipf_s: float = 0.0, cols: Sequence = (),
             permute_ids: bool = True, avoid_all_ones: bool = False) -> A.GenSpec:
    """cols: sequence of ("u32"|"i32"|"i64", lo, hi) uniform, ("normal",), ("ones",)."""
    sp = A.GenSpec()
    sp.seed = seed
    sp.key_bits = key_bits
    sp.ndv = ndv
    sp.zipf_s = zipf_s
    sp.permute_ids = int(permute_ids)
    sp.avoid_all_ones = int(avoid_all_ones)
    sp.ncols = len(cols)
    for i, c in enumerate(cols):
        kind = c[0]
        if kind == "normal":
            sp.col_kind[i] = A.GEN_NORMAL_F32
        elif kind == "ones":
            sp.col_kind[i] = A.GEN_ONES_I32
        else:
            sp.col_kind[i] = A.GEN_UNIFORM_I64 if kind == "i64" else A.GEN_UNIFORM_I32
            sp.col_lo[i], sp.col_hi[i] = int(c[1]), int(c[2])
    return sp


def _col_dtype(kind: int):
    return {A.GEN_UNIFORM_I32: np.int32, A.GEN_UNIFORM_I64: np.int64, A.GEN_NORMAL_F32: np.float32,
            A.GEN_ONES_I32: np.int32}[kind]


def gen_host(spec: A.GenSpec, n: int, row0: int = 0, nthreads: int = 8, key_unsigned: bool = False,
             out=None):
    """Generates rows [row0, row0+n) into numpy arrays (or the given ones)."""
    if out is None:
        kd = np.int64 if spec.key_bits == 64 else (np.uint32 if key_unsigned else np.int32)
        keys = np.empty(n, dtype=kd)
        cols = [np.empty(n, dtype=_col_dtype(spec.col_kind[i])) for i in range(spec.ncols)]
    else:
        keys, cols = out
    ptrs = (C.c_void_p * 4)(*([c.ctypes.data for c in cols] + [None] * (4 - len(cols))))
    A.check(A.lib().gba_gen_host(C.byref(spec), row0, n, C.c_void_p(keys.ctypes.data), ptrs, nthreads))
    return keys, cols


def gen_device(spec: A.GenSpec, n: int, row0: int = 0, device: int = 0, stream=None):
    import torch
    tmap = {np.int32: torch.int32, np.int64: torch.int64, np.float32: torch.float32}
    keys = torch.empty(n, dtype=torch.int64 if spec.key_bits == 64 else torch.int32, device=f"cuda:{device}")
    cols = [torch.empty(n, dtype=tmap[_col_dtype(spec.col_kind[i])], device=keys.device) for i in range(spec.ncols)]
    ptrs = (C.c_void_p * 4)(*([c.data_ptr() for c in cols] + [None] * (4 - len(cols))))
    s = stream if stream is not None else torch.cuda.current_stream(keys.device)
    A.check(A.lib().gba_gen_device(C.byref(spec), row0, n, C.c_void_p(keys.data_ptr()), ptrs,
                                   C.c_void_p(s.cuda_stream)))
    return keys, cols


# ---- serving ------------------------------------------------------------------------
@dataclass
class RequestInfo:
    ticket: int
    status: int
    n_groups: int
    lane: int
    batch_size: int
    queue_ms: float
    service_ms: float
    latency_ms: float


class Server:
    """Continuous-batching request loop over ``lanes`` CUDA streams
    (gba_server_*).  Requests take device tensors and device output buffers;
    keep both alive until the request is collected."""

    def __init__(self, device: int = 0, lanes: int = 4, memory_budget: int = 120 << 30, max_batch: int = 64,
                 batch_rows: int = 1 << 24, knobs=None, estimator_params=None):
        self._lib = A.lib()
        cfg = A.ServerConfig()
        self._lib.gba_server_default_config(C.byref(cfg))
        cfg.device, cfg.lanes, cfg.memory_budget = device, lanes, memory_budget
        cfg.max_batch, cfg.batch_rows = max_batch, batch_rows
        if knobs is not None:
            cfg.knobs = knobs if isinstance(knobs, A.Knobs) else make_knobs(**knobs)
        h = C.c_void_p()
        A.check(self._lib.gba_server_create(C.byref(h), C.byref(cfg)))
        self._h = h
        if estimator_params is not None:
            p = np.ascontiguousarray(estimator_params, dtype=np.float32)
            self._check(self._lib.gba_server_estimator_load(self._h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def _check(self, st):
        if st != A.OK:
            raise A.GbaError(st, f"{self._lib.gba_status_string(st).decode()} "
                                 f"({self._lib.gba_server_last_error(self._h).decode()})")

    def submit(self, keys, cols, aggs, out, unsigned_keys: bool = False) -> int:
        """out = (keys_out, [agg_out, ...]) device tensors (keys and keys_out
        pairs for a composite key); returns the ticket."""
        col_specs = [(c.data_ptr(), _torch_type(c)) for c in cols]
        k1, k2, uk = _split_keys(keys, unsigned_keys)
        q = build_query(k1.numel(), k1.data_ptr(), _torch_type(k1, uk[0]), col_specs, parse_aggs(aggs),
                        None if k2 is None else (k2.data_ptr(), _torch_type(k2, uk[1])))
        okeys, oaggs = out
        o = A.Output()
        for i, t in enumerate(oaggs):
            o.aggs[i] = t.data_ptr()
        o.capacity = _set_out_keys(o, okeys)
        t = C.c_int64(0)
        self._check(self._lib.gba_server_submit(self._h, C.byref(q), C.byref(o), C.byref(t)))
        return t.value

    @staticmethod
    def _info(ticket, i: A.RequestInfo) -> RequestInfo:
        return RequestInfo(ticket, i.status, i.n_groups, i.lane, i.batch_size, i.queue_ms, i.service_ms,
                           i.latency_ms)

    def wait(self, ticket: int, timeout: float = 60.0) -> RequestInfo:
        info = A.RequestInfo()
        self._check(self._lib.gba_server_wait(self._h, ticket, timeout, C.byref(info)))
        return self._info(ticket, info)

    def next_done(self, timeout: float = 0.0):
        """The next finished request, or None if none finished within timeout."""
        info = A.RequestInfo()
        t = C.c_int64(0)
        st = self._lib.gba_server_next_done(self._h, timeout, C.byref(t), C.byref(info))
        if st == A.ERR_TIMEOUT:
            return None
        self._check(st)
        return self._info(t.value, info)

    def pending(self):
        q, r, b = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        self._check(self._lib.gba_server_pending(self._h, C.byref(q), C.byref(r), C.byref(b)))
        return q.value, r.value, b.value

    def counters(self) -> dict:
        """Lane calls, failed batches, workspace releases, overflow reruns, and
        the longest lane call and release (ms) so far (gba_server_counters)."""
        n, f, rel, rg = C.c_int64(0), C.c_int64(0), C.c_int64(0), C.c_int64(0)
        lm, rm = C.c_double(0), C.c_double(0)
        self._check(self._lib.gba_server_counters(self._h, C.byref(n), C.byref(f), C.byref(rel), C.byref(rg),
                                                  C.byref(lm), C.byref(rm)))
        return {"lane_calls": n.value, "batch_failures": f.value, "ws_releases": rel.value, "regrows": rg.value,
                "lane_ms_max": round(lm.value, 3), "release_ms_max": round(rm.value, 3)}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gba_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
