"""ctypes mirror of ``include/gba.h`` and the loader of ``lib/libgba.so``.

The library is the product: there is no Python or CPU fallback.  Loading fails
loudly when the in-tree shared library is missing.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libgba.so"

GBA_MAX_COLS = 4
GBA_MAX_AGGS = 8
GBA_EST_FEATURES = 32
GBA_EST_HIDDEN = 64
GBA_EST_SAMPLE = 1024

# gba_status
OK, ERR_INVALID_ARG, ERR_CUDA, ERR_OOM, ERR_OUTPUT_CAPACITY, ERR_TABLE_OVERFLOW, ERR_TIMEOUT, ERR_UNSUPPORTED, \
    ERR_BUDGET = range(9)
# gba_type
I32, I64, F32, U32, F64 = 0, 1, 2, 3, 4
# gba_op
SUM, COUNT, MIN, MAX, AVG, COUNT_VALID = 0, 1, 2, 3, 4, 5
# gba_sizing
SIZING_PLAIN, SIZING_LEARNED, SIZING_FIXED, SIZING_GROW = 0, 1, 2, 3
# gba_strategy
STRATEGY_AUTO, STRATEGY_TABLE, STRATEGY_PARTITION = 0, 1, 2
# generator column kinds (csrc/datagen.h)
GEN_UNIFORM_I32, GEN_UNIFORM_I64, GEN_NORMAL_F32, GEN_ONES_I32 = 0, 1, 2, 3


class Column(C.Structure):
    _fields_ = [("type", C.c_int32), ("data", C.c_void_p), ("valid", C.c_void_p)]


class Agg(C.Structure):
    _fields_ = [("op", C.c_int32), ("col", C.c_int32)]


class Query(C.Structure):
    _fields_ = [
        ("n_rows", C.c_int64),
        ("key", Column),
        ("n_cols", C.c_int32),
        ("cols", Column * GBA_MAX_COLS),
        ("n_aggs", C.c_int32),
        ("aggs", Agg * GBA_MAX_AGGS),
        ("key2", Column),
    ]


class Output(C.Structure):
    _fields_ = [("keys", C.c_void_p), ("aggs", C.c_void_p * GBA_MAX_AGGS), ("capacity", C.c_int64),
                ("keys2", C.c_void_p), ("agg_valid", C.c_void_p * GBA_MAX_AGGS)]


class Knobs(C.Structure):
    _fields_ = [
        ("sizing", C.c_int32),
        ("strategy", C.c_int32),
        ("load_factor", C.c_double),
        ("table_slots", C.c_int64),
        ("preagg", C.c_int32),
        ("smem_slots", C.c_int32),
        ("partition_bits", C.c_int32),
        ("blocks_per_sm", C.c_int32),
        ("block_threads", C.c_int32),
        ("tile_rows", C.c_int32),
        ("nstages", C.c_int32),
        ("use_tma", C.c_int32),
        ("coalesce", C.c_int32),
        ("probe_cap", C.c_int32),
        ("smem_probe_cap", C.c_int32),
        ("max_regrow", C.c_int32),
        ("timing", C.c_int32),
        ("use_graph", C.c_int32),
        ("item_rows", C.c_int32),
        ("learned_load", C.c_double),
        ("learned_min_rows", C.c_int64),
        ("sort_output", C.c_int32),
        ("cluster_ctas", C.c_int32),
        ("exchange", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("strategy", C.c_int32),
        ("preagg", C.c_int32),
        ("table_slots", C.c_int64),
        ("partition_bits", C.c_int32),
        ("regrows", C.c_int32),
        ("predicted_groups", C.c_double),
        ("n_groups", C.c_int64),
        ("kernel_launches", C.c_int32),
        ("kernel_ms", C.c_double * 4),
        ("main_rows", C.c_int64),
        ("main_bytes", C.c_int64),
    ]


class GenSpec(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("key_bits", C.c_int),
        ("ndv", C.c_uint64),
        ("zipf_s", C.c_double),
        ("permute_ids", C.c_int),
        ("avoid_all_ones", C.c_int),
        ("ncols", C.c_int),
        ("col_kind", C.c_int * 4),
        ("col_lo", C.c_int64 * 4),
        ("col_hi", C.c_int64 * 4),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("lanes", C.c_int32),
        ("memory_budget", C.c_int64),
        ("max_batch", C.c_int32),
        ("batch_rows", C.c_int64),
        ("knobs", Knobs),
    ]


class RequestInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("lane", C.c_int32),
        ("batch_size", C.c_int32),
        ("n_groups", C.c_int64),
        ("queue_ms", C.c_double),
        ("service_ms", C.c_double),
        ("latency_ms", C.c_double),
    ]


# every function include/gba.h declares, with its ctypes signature
_P = C.c_void_p
SIGNATURES = {
    "gba_abi_struct_size": (C.c_int64, [C.c_int32]),
    "gba_default_knobs": (None, [C.POINTER(Knobs)]),
    "gba_status_string": (C.c_char_p, [C.c_int]),
    "gba_create": (C.c_int, [C.POINTER(_P), C.c_int32]),
    "gba_destroy": (C.c_int, [_P]),
    "gba_last_error": (C.c_char_p, [_P]),
    "gba_last_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "gba_groupby": (C.c_int, [_P, C.POINTER(Query), C.POINTER(Output), C.POINTER(Knobs), _P,
                              C.POINTER(C.c_int64)]),
    "gba_groupby_host": (C.c_int, [_P, C.POINTER(Query), C.POINTER(Output), C.POINTER(Knobs), _P,
                                   C.POINTER(C.c_int64)]),
    "gba_groupby_batch": (C.c_int, [_P, C.c_int32, C.POINTER(Query), C.POINTER(Output), C.POINTER(Knobs), _P,
                                    C.POINTER(C.c_int64)]),
    "gba_groupby_batch_host": (C.c_int, [_P, C.c_int32, C.POINTER(Query), C.POINTER(Output), C.POINTER(Knobs), _P,
                                         C.POINTER(C.c_int64)]),
    "gba_groupby_noalloc": (C.c_int, [_P, C.POINTER(Query), C.POINTER(Output), _P, C.POINTER(C.c_int64)]),
    "gba_groupby_partition_u32": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int32, _P, _P, _P, _P]),
    "gba_avg_divide": (C.c_int, [_P, C.c_int32, _P, C.POINTER(C.c_int32), _P, C.c_int64, _P]),
    "gba_autotune": (C.c_int, [_P, C.c_int32, C.POINTER(Query), C.POINTER(Output), C.POINTER(Knobs), _P, C.c_int32,
                               C.POINTER(Knobs), C.POINTER(C.c_double)]),
    "gba_server_default_config": (None, [C.POINTER(ServerConfig)]),
    "gba_server_create": (C.c_int, [C.POINTER(_P), C.POINTER(ServerConfig)]),
    "gba_server_estimator_load": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "gba_server_submit": (C.c_int, [_P, C.POINTER(Query), C.POINTER(Output), C.POINTER(C.c_int64)]),
    "gba_server_wait": (C.c_int, [_P, C.c_int64, C.c_double, C.POINTER(RequestInfo)]),
    "gba_server_next_done": (C.c_int, [_P, C.c_double, C.POINTER(C.c_int64), C.POINTER(RequestInfo)]),
    "gba_server_pending": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "gba_server_last_error": (C.c_char_p, [_P]),
    "gba_server_counters": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "gba_server_destroy": (C.c_int, [_P]),
    "gba_estimator_features": (C.c_int, [_P, C.POINTER(Query), C.c_int64, _P, C.POINTER(C.c_float)]),
    "gba_estimator_param_count": (C.c_int64, []),
    "gba_estimator_load": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "gba_estimator_get": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "gba_estimator_predict": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "gba_estimator_train": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32,
                                      C.c_int32, C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "gba_estimator_grad": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                     C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "gba_gen_host": (C.c_int, [C.POINTER(GenSpec), C.c_int64, C.c_int64, _P, C.POINTER(_P), C.c_int32]),
    "gba_gen_device": (C.c_int, [C.POINTER(GenSpec), C.c_int64, C.c_int64, _P, C.POINTER(_P), _P]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded ``libgba.so`` (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "or `python cpu_gpu_coprocess_groupby_agg_b200/build.py`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class GbaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gba status {status}: {message}")
        self.status = status


def check(status: int, ctx=None) -> None:
    if status != OK:
        L = lib()
        msg = L.gba_status_string(status).decode()
        if ctx is not None:
            detail = L.gba_last_error(ctx).decode()
            if detail:
                msg += f" ({detail})"
        raise GbaError(status, msg)
