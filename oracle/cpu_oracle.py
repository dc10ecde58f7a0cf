"""ctypes wrapper of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check in
__graft_entry__.py and by bench.py's CPU-baseline / reference leg.  The product
(libgba.so and its Python binding) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "liboracle.so"
REF_DRIVER = HERE / "_ref" / "ref_driver"

I32, I64, F32, U32, F64 = 0, 1, 2, 3, 4
SUM, COUNT, MIN, MAX, SUMABS = 0, 1, 2, 3, 4
_OPS = {"sum": SUM, "count": COUNT, "min": MIN, "max": MAX, "sumabs": SUMABS}

_lib = None


def build() -> None:
    """Builds lib/liboracle.so (and _ref/ref_driver where the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "-j8"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.orc_murmur3_32.restype = C.c_uint32
        L.orc_murmur3_32.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32]
        L.orc_groupby.restype = C.c_int64
        L.orc_groupby.argtypes = [C.c_int, C.c_void_p, C.c_int64, C.c_int, C.POINTER(C.c_int),
                                  C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_int]
        L.orc_tile_partition_counts.restype = None
        L.orc_tile_partition_counts.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p]
        L.orc_partition_of_u32.restype = C.c_uint32
        L.orc_partition_of_u32.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_partition_u32_array.restype = None
        L.orc_partition_u32_array.argtypes = [C.c_void_p, C.c_int64, C.c_uint32, C.c_void_p]
        L.orc_gen.restype = C.c_int
        L.orc_gen.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.POINTER(C.c_void_p), C.c_int]
        L.orc_merge_partitions.restype = C.c_int64
        L.orc_merge_partitions.argtypes = [C.c_void_p, C.c_int64, C.c_uint64, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _type(a: np.ndarray) -> int:
    return {np.dtype(np.int32): I32, np.dtype(np.uint32): U32, np.dtype(np.int64): I64,
            np.dtype(np.float32): F32, np.dtype(np.float64): F64}[a.dtype]


def murmur3_32(data: bytes, seed: int = 0) -> int:
    buf = C.create_string_buffer(data, len(data))
    return lib().orc_murmur3_32(buf, len(data), seed)


def groupby(keys: np.ndarray, cols=(), aggs=(("count", None),), nthreads: int = 1, sort: bool = True):
    """Exact GROUP BY; returns (keys, [agg arrays]) sorted by key.

    Integer aggregates are int64; SUM (and SUMABS) of fp32 and fp64 columns are float64.
    """
    keys = np.ascontiguousarray(keys)
    cols = [np.ascontiguousarray(c) for c in cols]
    n = keys.shape[0]
    ops = [_OPS[o] if isinstance(o, str) else int(o) for o, _ in aggs]
    acols = [0 if c is None else int(c) for _, c in aggs]
    ctypes_ = [_type(c) for c in cols]
    out_keys = np.empty(max(n, 1), dtype=keys.dtype)
    outs = []
    for o, c in zip(ops, acols):
        fp = o in (SUM, SUMABS) and o != COUNT and len(cols) > c and ctypes_[c] in (F32, F64)
        outs.append(np.empty(max(n, 1), dtype=np.float64 if fp else np.int64))
    na = len(ops)
    ct = (C.c_int * max(len(cols), 1))(*ctypes_)
    cp = (C.c_void_p * max(len(cols), 1))(*[c.ctypes.data for c in cols])
    op_arr = (C.c_int * na)(*ops)
    col_arr = (C.c_int * na)(*acols)
    op_ptrs = (C.c_void_p * na)(*[o.ctypes.data for o in outs])
    g = lib().orc_groupby(_type(keys), keys.ctypes.data, n, len(cols), ct, cp, na, op_arr, col_arr,
                          out_keys.ctypes.data, op_ptrs, nthreads, int(sort))
    return out_keys[:g], [o[:g] for o in outs]


def tile_partition_counts(keys_u32: np.ndarray, tile_len: int, P: int) -> np.ndarray:
    keys_u32 = np.ascontiguousarray(keys_u32, dtype=np.uint32)
    n = keys_u32.shape[0]
    nt = (n + tile_len - 1) // tile_len
    out = np.zeros((nt, P), dtype=np.uint32)
    lib().orc_tile_partition_counts(keys_u32.ctypes.data, n, tile_len, P, out.ctypes.data)
    return out


def partition_of_u32(keys_u32: np.ndarray, P: int) -> np.ndarray:
    """murmur3(key, seed 0) % P for every key (the reference's partition id)."""
    keys_u32 = np.ascontiguousarray(keys_u32, dtype=np.uint32)
    out = np.empty(keys_u32.shape[0], dtype=np.uint32)
    lib().orc_partition_u32_array(keys_u32.ctypes.data, keys_u32.shape[0], P, out.ctypes.data)
    return out


def merge_partitions(sizes: np.ndarray, K: int):
    sizes = np.ascontiguousarray(sizes, dtype=np.uint32)
    P = sizes.shape[0]
    merged_of = np.empty(P, dtype=np.int64)
    merged_sizes = np.empty(P, dtype=np.uint64)
    m = lib().orc_merge_partitions(sizes.ctypes.data, P, K, merged_of.ctypes.data, merged_sizes.ctypes.data)
    return merged_of, merged_sizes[:m]


def _mix64(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z ^= z >> np.uint64(31)
        z *= np.uint64(0x7FB5D329728EA185)
        z ^= z >> np.uint64(27)
        z *= np.uint64(0x81DADEF4BC2DD44D)
        z ^= z >> np.uint64(33)
    return z


def digest_pairs(keys: np.ndarray, vals: np.ndarray) -> str:
    """Order-independent digest of (u32 key, u32 value) pairs: sum of
    mix64(key << 32 | value) mod 2^64 - the digest oracle/ref_driver.cu writes."""
    z = (keys.astype(np.uint32).astype(np.uint64) << np.uint64(32)) | vals.astype(np.uint32).astype(np.uint64)
    with np.errstate(over="ignore"):
        return f"{int(_mix64(z).sum(dtype=np.uint64)):016x}"


_GEN_DTYPES = {0: np.int32, 1: np.int64, 2: np.float32, 3: np.int32}  # column kinds of datagen.h


def gen(spec, n: int, row0: int = 0, nthreads: int = 1, key_unsigned: bool = False):
    """Rows [row0, row0 + n) of a seeded generator spec (a ctypes structure with
    the layout of datagen.h's gba_gen_spec) as numpy (keys, [columns])."""
    kd = np.int64 if spec.key_bits == 64 else (np.uint32 if key_unsigned else np.int32)
    keys = np.empty(n, dtype=kd)
    cols = [np.empty(n, dtype=_GEN_DTYPES[spec.col_kind[i]]) for i in range(spec.ncols)]
    ptrs = (C.c_void_p * 4)(*([c.ctypes.data for c in cols] + [None] * (4 - len(cols))))
    rc = lib().orc_gen(C.addressof(spec), row0, n, keys.ctypes.data, ptrs, nthreads)
    if rc != 0:
        raise ValueError("orc_gen: bad generator spec")
    return keys, cols
