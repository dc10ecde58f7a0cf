"""The benchmark workloads, as seeded synthetic generator specs.

The reference publishes no dataset or benchmark; its driver generates keys with
std::rand (test/include/data_generator.hpp:7-105).  These five workloads are
the ones the project measures:

1. small: 2^20 rows, 32-bit keys uniform over 1,024 ids, int32 values in
   [0, 1000); SUM + COUNT.  Keys avoid 0xffffffff so the reference can run it.
2. skewed: 2^26 rows, int64 keys Zipf s=1.0 over 2^20 permuted ids; int64
   values uniform in [-2^31, 2^31) and fp32 values N(0,1); SUM/COUNT/MIN/MAX of
   the int64 column and SUM of the fp32 column.
3. high cardinality: 2^28 rows, int64 keys uniform over 2^26 ids; two int64
   columns uniform in [0, 2^20); SUM, SUM, COUNT.
4. batch: 256 queries, rows log-uniform in [2^12, 2^24], distinct ids
   log-uniform in [16, rows/2], Zipf s uniform in [0, 1.5], 32- or 64-bit keys
   (50/50), int64 values; SUM + COUNT.
5. serving: Poisson arrivals of batch-4-shaped queries plus 5% queries of
   2^27 rows over 2^24 int64 ids.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .api import gen_spec


@dataclass
class Workload:
    name: str
    n: int
    spec: object
    aggs: list
    key_unsigned: bool = False
    meta: dict = field(default_factory=dict)

    @property
    def key_bytes(self) -> int:
        return 8 if self.spec.key_bits == 64 else 4

    def col_bytes(self) -> list[int]:
        return [8 if self.spec.col_kind[i] == 1 else 4 for i in range(self.spec.ncols)]

    def row_bytes(self) -> int:
        return self.key_bytes + sum(self.col_bytes())

    def out_row_bytes(self) -> int:
        return self.key_bytes + 8 * len(self.aggs)


def small(seed: int = 1, n: int = 1 << 20, unsigned: bool = False) -> Workload:
    sp = gen_spec(seed, 32, 1024, 0.0, [("i32", 0, 1000)], permute_ids=True, avoid_all_ones=True)
    return Workload("small_2^20_uniform_1024", n, sp, [("sum", 0), ("count", None)], key_unsigned=unsigned)


def skewed(seed: int = 2, n: int = 1 << 26) -> Workload:
    sp = gen_spec(seed, 64, 1 << 20, 1.0, [("i64", -(1 << 31), 1 << 31), ("normal",)])
    return Workload("skewed_2^26_zipf1.0_2^20", n, sp,
                    [("sum", 0), ("count", None), ("min", 0), ("max", 0), ("sum", 1)])


def high_card(seed: int = 3, n: int = 1 << 28, ndv: int = 1 << 26) -> Workload:
    sp = gen_spec(seed, 64, ndv, 0.0, [("i64", 0, 1 << 20), ("i64", 0, 1 << 20)])
    return Workload(f"highcard_2^{int(math.log2(n))}_uniform_2^{int(math.log2(ndv))}", n, sp,
                    [("sum", 0), ("sum", 1), ("count", None)])


def batch_queries(seed: int = 4, count: int = 256, min_log2: float = 12.0, max_log2: float = 24.0) -> list[Workload]:
    """The mixed batch: shapes drawn from a seeded numpy generator."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(2 ** rng.uniform(min_log2, max_log2)))
        ndv = int(round(math.exp(rng.uniform(math.log(16), math.log(max(17, n // 2))))))
        s = float(rng.uniform(0.0, 1.5))
        bits = 64 if rng.random() < 0.5 else 32
        sp = gen_spec(seed * 1000003 + i, bits, ndv, s, [("i64", 0, 1 << 31)])
        out.append(Workload(f"q{i}", n, sp, [("sum", 0), ("count", None)], meta={"ndv": ndv, "zipf_s": s}))
    return out


def large_serving_query(seed: int) -> Workload:
    sp = gen_spec(seed, 64, 1 << 24, 0.0, [("i64", 0, 1 << 31)])
    return Workload("large_2^27_2^24", 1 << 27, sp, [("sum", 0), ("count", None)])
