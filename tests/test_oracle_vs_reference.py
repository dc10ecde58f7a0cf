"""Pins the oracle to the unmodified reference (CPU only).

tests/golden/ref_*.json were written by tests/golden/make_ref_fixtures.py, which
ran the reference itself (oracle/_ref/ref_driver, compiled from the reference
sources) on a B200.  Each fixture's input is regenerated bit-identically from
its generator parameters; the oracle must reproduce everything the reference
returned: the phase-1 partition sizes and (key, per-tile sum) digests, the
merged-partition layout (par_kv_begin / par_result_kv_num) and every merged
partition's (key, SUM) and (key, COUNT) pairs.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import cpu_oracle as O
from cpu_gpu_coprocess_groupby_agg_b200 import gen_host, gen_spec

GOLD = Path(__file__).parent / "golden"
FIXTURES = sorted(GOLD.glob("ref_*.json"))


def _input(fx):
    g = fx["generator"]
    sp = gen_spec(g["seed"], 32, g["ndv"], g["zipf_s"], [("i32", 0, 1000)], permute_ids=True, avoid_all_ones=True)
    keys, cols = gen_host(sp, g["n"], key_unsigned=True)
    return keys, cols[0].astype(np.uint32)


def _phase1(keys, vals, tile_len, P):
    """Per partition: sizes and digest of (key, per-tile aggregate) pairs."""
    sizes = np.zeros(P, dtype=np.int64)
    pk, pv = [[] for _ in range(P)], [[] for _ in range(P)]
    for t0 in range(0, len(keys), tile_len):
        k, (s,) = O.groupby(keys[t0:t0 + tile_len], [vals[t0:t0 + tile_len]], [("sum", 0)], nthreads=4)
        pid = O.partition_of_u32(k, P)
        order = np.argsort(pid, kind="stable")
        bounds = np.searchsorted(pid[order], np.arange(P + 1))
        for p in range(P):
            sl = order[bounds[p]:bounds[p + 1]]
            pk[p].append(k[sl])
            pv[p].append(s[sl].astype(np.uint32))
            sizes[p] += len(sl)
    digests = [O.digest_pairs(np.concatenate(pk[p]), np.concatenate(pv[p])) for p in range(P)]
    return sizes, digests


@pytest.mark.parametrize("path", FIXTURES, ids=[p.stem for p in FIXTURES])
def test_oracle_reproduces_reference(path):
    fx = json.loads(path.read_text())
    keys, vals = _input(fx)
    assert len(keys) == fx["generator"]["n"]
    tile_len, P, cap = fx["tile_len"], fx["P"], fx["capacity"]
    for agg, v in (("sum", vals), ("count", np.ones_like(vals))):
        ref = fx[agg]
        sizes, digests = _phase1(keys, v, tile_len, P)
        assert sizes.tolist() == ref["phase1_sizes"], f"{agg}: phase-1 partition sizes"
        assert digests == ref["phase1_digests"], f"{agg}: phase-1 partition contents"
        # phase 2 layout: greedy merge up to min_load_num = 3/5 Capacity
        merged_of, merged_sizes = O.merge_partitions(sizes.astype(np.uint32), cap * 3 // 5)
        begin = np.concatenate([[0], np.cumsum(merged_sizes)[:-1]]).astype(np.int64)
        assert begin.tolist() == ref["par_kv_begin"], f"{agg}: par_kv_begin"
        # final groups, placed in the merged partition their partition joined
        k, (s,) = O.groupby(keys, [v], [("sum", 0)], nthreads=4)
        mp = merged_of[O.partition_of_u32(k, P)]
        kv_num = np.bincount(mp, minlength=len(merged_sizes))
        assert kv_num.tolist() == ref["par_result_kv_num"], f"{agg}: par_result_kv_num"
        got = [O.digest_pairs(k[mp == i], s[mp == i].astype(np.uint32)) for i in range(len(merged_sizes))]
        assert got == ref["merged_digests"], f"{agg}: merged partition results"
        assert O.digest_pairs(k, s.astype(np.uint32)) == ref["result_digest"]
        assert len(k) == ref["groups"] == ref["distinct_keys_in_output"]
        if "sorted_keys" in ref:
            assert k.tolist() == ref["sorted_keys"]
            assert s.astype(np.uint32).tolist() == ref["sorted_values"]


def test_fixtures_present():
    names = {p.stem for p in FIXTURES}
    assert {"ref_small_uniform_1024", "ref_highcard_uniform_2e19", "ref_zipf0.9_100k_ragged",
            "ref_one_tile_p1024"} <= names
