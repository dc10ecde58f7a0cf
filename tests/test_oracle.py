"""The oracle is pinned before it is trusted (CPU only).

* MurmurHash3_x86_32 against independent known answers (tests/golden/murmur3_kat.json).
* orc_groupby against a numpy restatement of exact GROUP BY, every type/aggregate.
* The reference's phase-1 layout (per-tile distinct keys, murmur(k,0) % P) and its
  greedy partition merge against numpy / property checks.
* Fixtures produced by running the unmodified reference (tests/golden/ref_*.json).
"""
import json
from pathlib import Path

import numpy as np
import pytest

import cpu_oracle as O

GOLD = Path(__file__).parent / "golden"


def test_murmur3_known_answers():
    cases = json.loads((GOLD / "murmur3_kat.json").read_text())
    assert len(cases) >= 100
    for c in cases:
        assert O.murmur3_32(bytes.fromhex(c["bytes"]), c["seed"]) == c["hash"], c


def _np_groupby(keys, cols, aggs):
    uk, inv = np.unique(keys, return_inverse=True)
    outs = []
    for op, c in aggs:
        if op == "count":
            outs.append(np.bincount(inv, minlength=len(uk)).astype(np.int64))
            continue
        x = cols[c]
        if x.dtype == np.float32:
            acc = np.zeros(len(uk), dtype=np.float64)
            np.add.at(acc, inv, x.astype(np.float64))
        elif op == "sum":
            acc = np.zeros(len(uk), dtype=np.int64)
            np.add.at(acc, inv, x.astype(np.int64))
        elif op == "min":
            acc = np.full(len(uk), np.iinfo(np.int64).max, dtype=np.int64)
            np.minimum.at(acc, inv, x.astype(np.int64))
        else:
            acc = np.full(len(uk), np.iinfo(np.int64).min, dtype=np.int64)
            np.maximum.at(acc, inv, x.astype(np.int64))
        outs.append(acc)
    return uk, outs


@pytest.mark.parametrize("kdt", [np.int32, np.uint32, np.int64])
@pytest.mark.parametrize("nthreads", [1, 4])
def test_groupby_matches_numpy(kdt, nthreads):
    rng = np.random.default_rng(7)
    n = 200_000
    if kdt == np.int64:
        dom = rng.integers(-(1 << 62), 1 << 62, size=5000, dtype=np.int64)
    else:
        info = np.iinfo(kdt)
        dom = rng.integers(info.min, int(info.max) + 1, size=5000, dtype=np.int64).astype(kdt)
    keys = dom[rng.integers(0, len(dom), size=n)]
    cols = [rng.integers(-(1 << 40), 1 << 40, size=n, dtype=np.int64),
            rng.integers(-1000, 1000, size=n, dtype=np.int32).astype(np.int32),
            rng.standard_normal(n).astype(np.float32),
            rng.integers(0, 1 << 31, size=n, dtype=np.int64).astype(np.uint32)]
    aggs = [("sum", 0), ("count", None), ("min", 0), ("max", 0), ("sum", 1), ("min", 1), ("sum", 2), ("sum", 3)]
    k, outs = O.groupby(keys, cols, aggs, nthreads=nthreads)
    ek, eouts = _np_groupby(keys, cols, aggs)
    np.testing.assert_array_equal(k, ek)
    for a, (o, e) in enumerate(zip(outs, eouts)):
        if o.dtype == np.float64:
            np.testing.assert_allclose(o, e, rtol=1e-12, atol=1e-9)
        else:
            np.testing.assert_array_equal(o, e, err_msg=str(aggs[a]))


def test_groupby_edge_cases():
    k, outs = O.groupby(np.zeros(0, dtype=np.int64), [], [("count", None)])
    assert len(k) == 0
    keys = np.array([-1, -1, 0, np.iinfo(np.int64).min, np.iinfo(np.int64).max, -1], dtype=np.int64)
    v = np.array([1, 2, 3, 4, 5, 6], dtype=np.int64)
    k, outs = O.groupby(keys, [v], [("sum", 0), ("count", None), ("max", 0)])
    assert list(k) == [np.iinfo(np.int64).min, -1, 0, np.iinfo(np.int64).max]
    assert list(outs[0]) == [4, 9, 3, 5]
    assert list(outs[1]) == [1, 3, 1, 1]
    # u32 all-ones key (the reference's empty marker) is an ordinary key here
    keys = np.array([0xFFFFFFFF, 0xFFFFFFFF, 7], dtype=np.uint32)
    k, outs = O.groupby(keys, [np.array([1, 2, 3], dtype=np.uint32)], [("sum", 0)])
    assert list(k) == [7, 0xFFFFFFFF] and list(outs[0]) == [3, 3]


def test_f64_sum_matches_fsum():
    """fp64 value columns: each group's SUM within a few roundings of the
    correctly rounded sum (math.fsum), SUMABS likewise."""
    import math
    rng = np.random.default_rng(3)
    n = 50_000
    keys = rng.integers(0, 300, size=n).astype(np.int64)
    v = rng.standard_normal(n) * 10.0 ** rng.integers(-20, 20, size=n)
    k, (s, a) = O.groupby(keys, [v], [("sum", 0), ("sumabs", 0)], nthreads=4)
    for i, key in enumerate(k):
        x = v[keys == key]
        assert abs(s[i] - math.fsum(x)) <= 1e-12 * math.fsum(np.abs(x))
        assert abs(a[i] - math.fsum(np.abs(x))) <= 1e-12 * math.fsum(np.abs(x))


def test_sum_wraps_mod_2_64():
    keys = np.zeros(3, dtype=np.int64)
    v = np.array([np.iinfo(np.int64).max, 1, 1], dtype=np.int64)
    _, outs = O.groupby(keys, [v], [("sum", 0)])
    assert outs[0][0] == np.iinfo(np.int64).min + 1


def test_tile_partition_counts_match_numpy():
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 3000, size=50_000, dtype=np.int64).astype(np.uint32)
    tile, P = 12_000, 300
    got = O.tile_partition_counts(keys, tile, P)
    for t in range(got.shape[0]):
        uk = np.unique(keys[t * tile:(t + 1) * tile])
        pid = O.partition_of_u32(uk, P)
        np.testing.assert_array_equal(got[t], np.bincount(pid, minlength=P))


def test_merge_partitions_properties():
    rng = np.random.default_rng(5)
    sizes = rng.integers(0, 5000, size=300).astype(np.uint32)
    K = 60_000
    of, ms = O.merge_partitions(sizes, K)
    assert ms.sum() == sizes.sum()
    for m in range(len(ms)):
        assert ms[m] == sizes[of == m].sum()
        if (of == m).sum() > 1:
            assert ms[m] <= K
    # no two remaining merged partitions could still be merged (greedy fixpoint)
    srt = np.sort(ms)
    assert len(ms) == 1 or srt[0] + srt[1] > K


def test_generator_properties():
    from cpu_gpu_coprocess_groupby_agg_b200 import gen_host, gen_spec
    sp = gen_spec(11, 64, 1000, 1.0, [("i64", -5, 5), ("normal",), ("i32", 0, 1000)], permute_ids=False)
    k, cols = gen_host(sp, 400_000, nthreads=4)
    assert k.min() >= 0 and k.max() < 1000
    counts = np.bincount(k, minlength=1000)
    # Zipf s=1: P(rank 1) / P(rank 2) == 2
    assert 1.85 < counts[0] / counts[1] < 2.15
    assert cols[0].min() >= -5 and cols[0].max() < 5
    assert abs(float(cols[1].mean())) < 0.01 and abs(float(cols[1].std()) - 1) < 0.01
    assert cols[2].min() >= 0 and cols[2].max() < 1000
    # slices are independent of the split
    k2, c2 = gen_host(sp, 1000, row0=12345, nthreads=1)
    np.testing.assert_array_equal(k2, k[12345:13345])
    np.testing.assert_array_equal(c2[1], cols[1][12345:13345])
    # uniform over a permuted domain: exactly ndv distinct keys, never all-ones
    sp = gen_spec(1, 32, 1024, 0.0, [("i32", 0, 1000)], avoid_all_ones=True)
    k, _ = gen_host(sp, 1 << 16, key_unsigned=True)
    assert len(np.unique(k)) == 1024 and not (k == 0xFFFFFFFF).any()


def test_oracle_generator_matches_the_library_generator():
    """The reference arm of the benchmark generates its inputs with the
    oracle's copy of the generator (it must not load the library); both must
    give the same bytes."""
    from cpu_gpu_coprocess_groupby_agg_b200 import gen_host, gen_spec, workloads as W
    specs = [gen_spec(11, 64, 1000, 1.0, [("i64", -5, 5), ("normal",), ("i32", 0, 1000)], permute_ids=False),
             gen_spec(1, 32, 1024, 0.0, [("i32", 0, 1000)], avoid_all_ones=True),
             gen_spec(7, 32, 300_000, 1.45, [("i64", 0, 1 << 31)])]
    specs += [q.spec for q in W.batch_queries()[:6]]
    for sp in specs:
        for row0, n, th in ((0, 70_000, 4), (123_457, 5000, 1)):
            k1, c1 = gen_host(sp, n, row0=row0, nthreads=th)
            k2, c2 = O.gen(sp, n, row0=row0, nthreads=3)
            assert k1.dtype == k2.dtype
            np.testing.assert_array_equal(k1, k2)
            for a, b in zip(c1, c2):
                assert a.dtype == b.dtype
                np.testing.assert_array_equal(a, b)
