"""Generates murmur3_kat.json: MurmurHash3_x86_32 known answers.

The answers come from scikit-learn's ``sklearn.utils.murmurhash3_32`` (an
independent implementation of the published algorithm, used as a black box).
They pin the oracle's hash (oracle/oracle.cpp), the device hash used by the
kernels and the cuco stand-in used to build the reference.  Run in an
environment with scikit-learn:  python tests/golden/make_murmur3_kat.py
"""
import json
import struct
from pathlib import Path

from sklearn.utils import murmurhash3_32

cases = []
for seed in (0, 1, 42, 0x9747B28C, 0xFFFFFFFF):
    for k in (0, 1, 2, 3, 255, 256, 1 << 16, 0x7FFFFFFF, 0x80000000, 0xFFFFFFFE, 0xFFFFFFFF, 123456789, 3735928559):
        b = struct.pack("<I", k)
        cases.append({"bytes": b.hex(), "seed": seed, "hash": murmurhash3_32(b, seed=seed & 0xFFFFFFFF, positive=True)})
    for k in (0, 1, -1, 1 << 40, (1 << 63) - 1, -(1 << 63), 0x0123456789ABCDEF, 1099511627781):
        b = struct.pack("<q", k)
        cases.append({"bytes": b.hex(), "seed": seed, "hash": murmurhash3_32(b, seed=seed & 0xFFFFFFFF, positive=True)})
    for s in (b"", b"a", b"ab", b"abc", b"hello world"):
        cases.append({"bytes": s.hex(), "seed": seed, "hash": murmurhash3_32(s, seed=seed & 0xFFFFFFFF, positive=True)})
Path(__file__).with_name("murmur3_kat.json").write_text(json.dumps(cases, indent=0))
print(len(cases), "cases")
