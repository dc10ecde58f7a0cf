"""Runs the UNMODIFIED reference (oracle/_ref/ref_driver, built by oracle/Makefile
from the reference sources) on seeded u32 inputs and records what it returns
as fixtures ``ref_<case>.json``.  Needs a CUDA GPU.

For every case the reference runs twice, exactly as its own driver calls it
(test/test.cu:134-161): once with the value column (GROUP BY SUM) and once
with all values 1 (which makes its SUM a COUNT).  A fixture holds the inputs'
generator parameters (the input is regenerated bit-identically from them),
the phase-1 partition sizes and pair digests, the merged-partition layout
(par_kv_begin / par_result_kv_num), a digest of every merged partition's
(key, sum) pairs and, for small outputs, the sorted result itself.

  python tests/golden/make_ref_fixtures.py --out tests/golden
"""
import argparse
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from cpu_gpu_coprocess_groupby_agg_b200 import gen_host, gen_spec  # noqa: E402

DRIVER = ROOT / "oracle" / "_ref" / "ref_driver"

# name: (seed, n, ndv, zipf_s, tile_len, P, nstreams)
CASES = {
    "small_uniform_1024": (1, 1 << 20, 1024, 0.0, 1 << 18, 300, 4),
    "highcard_uniform_2e19": (21, 1 << 20, 1 << 19, 0.0, 1 << 18, 300, 4),
    "zipf0.9_100k_ragged": (22, 1_000_003, 100_000, 0.9, 1 << 18, 300, 4),
    "one_tile_p1024": (23, 300_000, 20_000, 0.0, 1 << 19, 1024, 2),
}


def spec_of(seed, ndv, zipf_s):
    return gen_spec(seed, 32, ndv, zipf_s, [("i32", 0, 1000)], permute_ids=True, avoid_all_ones=True)


def make_input(seed, n, ndv, zipf_s):
    keys, cols = gen_host(spec_of(seed, ndv, zipf_s), n, key_unsigned=True, nthreads=8)
    return keys, cols[0].astype(np.uint32)


def mix64(z):
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z ^= z >> np.uint64(31)
        z *= np.uint64(0x7FB5D329728EA185)
        z ^= z >> np.uint64(27)
        z *= np.uint64(0x81DADEF4BC2DD44D)
        z ^= z >> np.uint64(33)
    return z


def digest_pairs(keys, vals) -> str:
    z = (keys.astype(np.uint64) << np.uint64(32)) | vals.astype(np.uint32).astype(np.uint64)
    with np.errstate(over="ignore"):
        return f"{int(mix64(z).sum(dtype=np.uint64)):016x}"


def run_driver(keys, vals, tile_len, P, nstreams, workdir: Path, tag: str):
    inp = workdir / f"{tag}.in"
    with open(inp, "wb") as f:
        f.write(np.int64(len(keys)).tobytes())
        f.write(keys.astype(np.uint32).tobytes())
        f.write(vals.astype(np.uint32).tobytes())
    outp = workdir / tag
    subprocess.run([str(DRIVER), str(inp), str(outp), str(tile_len), str(P), str(nstreams), str(tile_len)],
                   check=True, timeout=600)
    meta = json.loads(Path(str(outp) + ".json").read_text())
    raw = Path(str(outp) + ".bin").read_bytes()
    parts = []
    off = 0
    while off < len(raw):
        m = int(np.frombuffer(raw, dtype=np.uint64, count=1, offset=off)[0])
        off += 8
        k = np.frombuffer(raw, dtype=np.uint32, count=m, offset=off)
        off += 4 * m
        v = np.frombuffer(raw, dtype=np.uint32, count=m, offset=off)
        off += 4 * m
        parts.append((k.copy(), v.copy()))
    return meta, parts


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).parent))
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for name, (seed, n, ndv, zipf_s, tile_len, P, nstreams) in CASES.items():
            keys, vals = make_input(seed, n, ndv, zipf_s)
            fx = {"case": name, "generator": {"seed": seed, "n": n, "ndv": ndv, "zipf_s": zipf_s, "key_bits": 32,
                                              "value": "uniform int32 [0,1000)", "avoid_all_ones": True},
                  "tile_len": tile_len, "P": P, "nstreams": nstreams, "capacity": tile_len}
            for agg, v in (("sum", vals), ("count", np.ones_like(vals))):
                meta, parts = run_driver(keys, v, tile_len, P, nstreams, td, f"{name}_{agg}")
                allk = np.concatenate([p[0] for p in parts])
                allv = np.concatenate([p[1] for p in parts])
                fx[agg] = {
                    "phase1_sizes": meta["phase1_sizes"],
                    "phase1_digests": meta["phase1_digests"],
                    "par_kv_begin": meta["par_kv_begin"],
                    "par_result_kv_num": meta["par_result_kv_num"],
                    "merged_digests": [digest_pairs(k, vv) for k, vv in parts],
                    "groups": int(len(allk)),
                    "distinct_keys_in_output": int(len(np.unique(allk))),
                    "result_digest": digest_pairs(allk, allv),
                    "phase1_s": meta["phase1_s"], "phase2_s": meta["phase2_s"],
                }
                if len(allk) <= 4096:
                    o = np.argsort(allk)
                    fx[agg]["sorted_keys"] = allk[o].tolist()
                    fx[agg]["sorted_values"] = allv[o].tolist()
            (out / f"ref_{name}.json").write_text(json.dumps(fx))
            print(name, fx["sum"]["groups"], "groups,", len(fx["sum"]["par_kv_begin"]), "merged partitions,",
                  f"phase1 {fx['sum']['phase1_s']:.4f}s phase2 {fx['sum']['phase2_s']:.4f}s")


if __name__ == "__main__":
    main()
