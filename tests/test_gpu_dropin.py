"""The drop-in C++ API (include/tiled_groupby_agg_partition.hpp) against the
reference's own outputs and the oracle.

lib/tiled_driver calls groupby_agg_partition<u32,u32> and
groupby_agg_intra_partition exactly as the reference's test/test.cu does.  On
every golden case (tests/golden/ref_*.json, written by running the unmodified
reference) it must return what the reference returned: the phase-1 partition
sizes and (key, per-tile sum) digests, par_kv_begin, par_result_kv_num and
every merged partition's (key, SUM) pairs - for the value column and for
all-ones values (COUNT).  Cases the reference cannot run (the key 0xffffffff,
P = 1, more workers than tiles, an empty input) are checked against the oracle.
gba_groupby_partition_u32, the C ABI under it, is checked per tile.
"""
import ctypes as C
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

import cpu_oracle as O
from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
from cpu_gpu_coprocess_groupby_agg_b200 import gen_host, gen_spec

GOLD = Path(__file__).parent / "golden"
FIXTURES = sorted(GOLD.glob("ref_*.json"))
DRIVER = A.LIB_PATH.parent / "tiled_driver"


def _fixture_input(g):
    sp = gen_spec(g["seed"], 32, g["ndv"], g["zipf_s"], [("i32", 0, 1000)], permute_ids=True, avoid_all_ones=True)
    keys, cols = gen_host(sp, g["n"], key_unsigned=True)
    return keys.view(np.uint32), cols[0].astype(np.uint32)


def run_driver(tmp: Path, keys, vals, tile_len, P, nstreams, capacity, tag="run"):
    inp = tmp / f"{tag}.in"
    with open(inp, "wb") as f:
        f.write(np.int64(len(keys)).tobytes())
        f.write(keys.astype(np.uint32).tobytes())
        f.write(vals.astype(np.uint32).tobytes())
    outp = tmp / tag
    r = subprocess.run([str(DRIVER), str(inp), str(outp), str(tile_len), str(P), str(nstreams), str(capacity)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    meta = json.loads(Path(str(outp) + ".json").read_text())
    raw = Path(str(outp) + ".bin").read_bytes()
    parts, off = [], 0
    while off < len(raw):
        m = int(np.frombuffer(raw, dtype=np.uint64, count=1, offset=off)[0])
        off += 8
        k = np.frombuffer(raw, dtype=np.uint32, count=m, offset=off).copy()
        off += 4 * m
        v = np.frombuffer(raw, dtype=np.uint32, count=m, offset=off).copy()
        off += 4 * m
        parts.append((k, v))
    return meta, parts


def oracle_expect(keys, vals, tile_len, P, capacity):
    """What the reference computes, restated by the oracle (phase 1 per tile,
    greedy merge, final groups per merged partition)."""
    sizes = np.zeros(P, dtype=np.int64)
    pk, pv = [[] for _ in range(P)], [[] for _ in range(P)]
    for t0 in range(0, len(keys), tile_len):
        k, (s,) = O.groupby(keys[t0:t0 + tile_len], [vals[t0:t0 + tile_len]], [("sum", 0)], nthreads=4)
        pid = O.partition_of_u32(k, P)
        for p in range(P):
            sel = pid == p
            pk[p].append(k[sel])
            pv[p].append(s[sel].astype(np.uint32))
            sizes[p] += int(sel.sum())
    digests = [O.digest_pairs(np.concatenate(pk[p]) if pk[p] else np.zeros(0, np.uint32),
                              np.concatenate(pv[p]) if pv[p] else np.zeros(0, np.uint32)) for p in range(P)]
    merged_of, merged_sizes = O.merge_partitions(sizes.astype(np.uint32), capacity * 3 // 5)
    begin = np.concatenate([[0], np.cumsum(merged_sizes)[:-1]]).astype(np.int64)
    k, (s,) = O.groupby(keys, [vals], [("sum", 0)], nthreads=4)
    mp = merged_of[O.partition_of_u32(k, P)]
    kv_num = np.bincount(mp, minlength=len(merged_sizes))
    merged = [O.digest_pairs(k[mp == i], s[mp == i].astype(np.uint32)) for i in range(len(merged_sizes))]
    return {"phase1_sizes": sizes.tolist(), "phase1_digests": digests, "par_kv_begin": begin.tolist(),
            "par_result_kv_num": kv_num.tolist(), "merged_digests": merged,
            "result_digest": O.digest_pairs(k, s.astype(np.uint32)), "groups": len(k)}


def check(meta, parts, want, label):
    assert meta["segments_in_place"], f"{label}: phase-1 segments do not point at their own tiles"
    assert meta["phase1_sizes"] == want["phase1_sizes"], f"{label}: phase-1 partition sizes"
    assert meta["phase1_digests"] == want["phase1_digests"], f"{label}: phase-1 partition contents"
    assert meta["par_kv_begin"] == want["par_kv_begin"], f"{label}: par_kv_begin"
    assert meta["par_result_kv_num"] == want["par_result_kv_num"], f"{label}: par_result_kv_num"
    got = [O.digest_pairs(k, v) for k, v in parts]
    assert got == want["merged_digests"], f"{label}: merged partition results"
    allk = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, np.uint32)
    allv = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0, np.uint32)
    assert len(allk) == want["groups"] == len(np.unique(allk)), f"{label}: group count"
    assert O.digest_pairs(allk, allv) == want["result_digest"], f"{label}: result"


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[p.stem for p in FIXTURES])
def test_dropin_matches_reference_fixture(path, tmp_path):
    fx = json.loads(path.read_text())
    keys, vals = _fixture_input(fx["generator"])
    for agg, v in (("sum", vals), ("count", np.ones_like(vals))):
        meta, parts = run_driver(tmp_path, keys, v, fx["tile_len"], fx["P"], fx["nstreams"], fx["capacity"], agg)
        check(meta, parts, fx[agg], f"{path.stem}/{agg}")
        if "sorted_keys" in fx[agg]:
            allk = np.concatenate([p[0] for p in parts])
            allv = np.concatenate([p[1] for p in parts])
            o = np.argsort(allk)
            assert allk[o].tolist() == fx[agg]["sorted_keys"]
            assert allv[o].tolist() == fx[agg]["sorted_values"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["empty_key_ragged", "p1_many_workers", "wrapping_sums", "empty_input", "p4096"])
def test_dropin_against_oracle(case, tmp_path):
    rng = np.random.default_rng(7)
    if case == "empty_key_ragged":
        # 0xffffffff is the reference's empty marker (util.cuh:8); here it is a key
        n, tile, P, ns, cap = 250_001, 65_536, 300, 4, 65_536
        keys = rng.integers(0, 5000, n, dtype=np.uint64).astype(np.uint32)
        keys[rng.random(n) < 0.01] = 0xFFFFFFFF
        vals = rng.integers(0, 1000, n, dtype=np.uint64).astype(np.uint32)
    elif case == "p1_many_workers":
        n, tile, P, ns, cap = 100_000, 40_000, 1, 8, 100_000
        keys = rng.integers(0, 70_000, n, dtype=np.uint64).astype(np.uint32)
        vals = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    elif case == "wrapping_sums":
        # per-key sums far above 2^32: the u32 result wraps like the reference's
        n, tile, P, ns, cap = 200_000, 50_000, 64, 3, 50_000
        keys = rng.integers(0, 8, n, dtype=np.uint64).astype(np.uint32)
        vals = rng.integers(1 << 31, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    elif case == "empty_input":
        n, tile, P, ns, cap = 0, 1024, 16, 2, 1024
        keys = np.zeros(0, np.uint32)
        vals = np.zeros(0, np.uint32)
    else:  # fan-out beyond the reference's 1024
        n, tile, P, ns, cap = 300_000, 1 << 17, 4096, 4, 1 << 17
        keys = rng.integers(0, 200_000, n, dtype=np.uint64).astype(np.uint32)
        vals = rng.integers(0, 1000, n, dtype=np.uint64).astype(np.uint32)
    if n == 0:
        meta, parts = run_driver(tmp_path, keys, vals, tile, P, ns, cap)
        assert meta["phase1_sizes"] == [0] * P
        assert sum(meta["par_result_kv_num"]) == 0
        return
    want = oracle_expect(keys, vals, tile, P, cap)
    meta, parts = run_driver(tmp_path, keys, vals, tile, P, ns, cap)
    check(meta, parts, want, case)


@pytest.mark.gpu
@pytest.mark.parametrize("P", [1, 7, 300, 1024, 16384])
def test_groupby_partition_u32_layout(ctx, P):
    """One tile through the C ABI: partition-ordered groups and offsets."""
    import torch
    rng = np.random.default_rng(P)
    n = 123_457
    keys = rng.integers(0, 40_000, n, dtype=np.uint64).astype(np.uint32)
    keys[::97] = 0xFFFFFFFF
    vals = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    dk = torch.from_numpy(keys.view(np.int32)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    ok = torch.empty(n, dtype=torch.int32, device="cuda")
    ov = torch.empty(n, dtype=torch.int32, device="cuda")
    offs = np.zeros(P + 1, dtype=np.uint64)
    st = A.lib().gba_groupby_partition_u32(ctx.handle, dk.data_ptr(), dv.data_ptr(), n, P, ok.data_ptr(),
                                           ov.data_ptr(), offs.ctypes.data, torch.cuda.current_stream().cuda_stream)
    A.check(st, ctx.handle)
    k, (s,) = O.groupby(keys, [vals], [("sum", 0)], nthreads=4)
    g = int(offs[P])
    assert g == len(k)
    gk = ok[:g].cpu().numpy().view(np.uint32)
    gv = ov[:g].cpu().numpy().view(np.uint32)
    pid = O.partition_of_u32(k, P)
    want_sizes = np.bincount(pid, minlength=P)
    assert np.array_equal(np.diff(offs.astype(np.int64)), want_sizes)
    for p in range(0, P, max(1, P // 64)):
        a, b = int(offs[p]), int(offs[p + 1])
        sel = pid == p
        assert O.digest_pairs(gk[a:b], gv[a:b]) == O.digest_pairs(k[sel], s[sel].astype(np.uint32)), p
    assert O.digest_pairs(gk, gv) == O.digest_pairs(k, s.astype(np.uint32))


@pytest.mark.gpu
def test_groupby_partition_u32_in_place(ctx):
    """Output over the input, as phase 1 writes a tile's groups over itself."""
    import torch
    rng = np.random.default_rng(3)
    n = 77_777
    keys = rng.integers(0, 9_000, n, dtype=np.uint64).astype(np.uint32)
    vals = rng.integers(0, 1000, n, dtype=np.uint64).astype(np.uint32)
    dk = torch.from_numpy(keys.view(np.int32)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    P = 300
    offs = np.zeros(P + 1, dtype=np.uint64)
    st = A.lib().gba_groupby_partition_u32(ctx.handle, dk.data_ptr(), dv.data_ptr(), n, P, dk.data_ptr(),
                                           dv.data_ptr(), offs.ctypes.data, torch.cuda.current_stream().cuda_stream)
    A.check(st, ctx.handle)
    k, (s,) = O.groupby(keys, [vals], [("sum", 0)], nthreads=4)
    g = int(offs[P])
    assert g == len(k)
    assert O.digest_pairs(dk[:g].cpu().numpy().view(np.uint32), dv[:g].cpu().numpy().view(np.uint32)) == \
        O.digest_pairs(k, s.astype(np.uint32))


def test_partition_u32_rejects_bad_fanout():
    """Argument checks need no GPU: P outside [1, 16384] is refused."""
    h = C.c_void_p()
    # without a device the context cannot be created; with one, it can
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if not have_gpu:
        assert A.lib().gba_groupby_partition_u32(None, None, None, 0, 1, None, None, None, None) == A.ERR_INVALID_ARG
        return
    A.check(A.lib().gba_create(C.byref(h), 0))
    offs = np.zeros(2, dtype=np.uint64)
    for P in (0, 16385):
        assert A.lib().gba_groupby_partition_u32(h, None, None, 0, P, None, None, offs.ctypes.data, None) == \
            A.ERR_INVALID_ARG
    A.lib().gba_destroy(h)
