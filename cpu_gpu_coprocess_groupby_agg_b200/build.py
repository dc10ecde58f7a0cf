"""Build recipe for the in-tree shared library ``lib/libgba.so`` (sm_100a).

Every ``csrc/*.cu`` file is compiled by nvcc for ``sm_100a`` only and linked
into one shared library with the CUDA runtime linked statically, so the
library loads on any host (a GPU is needed only to run kernels).  Objects are
cached under ``_build/`` and rebuilt when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
BUILD = PKG.parent / "_build" / "gba"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-Wall",
    "--expt-relaxed-constexpr",
    "-I", str(INCLUDE),
    "-I", str(CSRC),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libgba.so")


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h*")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, extra: list[str]) -> str:
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile (incrementally) and link ``lib/libgba.so``; returns its path."""
    BUILD.mkdir(parents=True, exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    headers = _headers()
    objs = []
    todo = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if _stale(obj, [src, *headers]):
            todo.append((src, obj))
    extra = ["-Xptxas", "-v"] if verbose else []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 2)) as ex:
        futs = {ex.submit(_compile, s, o, extra): s for s, o in todo}
        for f in cf.as_completed(futs):
            log = f.result()
            if verbose and log:
                print(f"== {futs[f].name}\n{log}", file=sys.stderr)
    lib = LIBDIR / "libgba.so"
    if _stale(lib, objs) or todo:
        # linked beside the library and renamed over it, so a reader never sees a partial file
        tmp = LIBDIR / f".libgba.so.{os.getpid()}"
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs), "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            tmp.unlink(missing_ok=True)
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, lib)
    build_driver(lib)
    return lib


DRIVER_SRC = PKG.parent / "tests" / "drivers" / "tiled_driver.cu"


def build_driver(lib: Path) -> Path | None:
    """``lib/tiled_driver``: a caller of the drop-in C++ API written like the
    reference's test/test.cu (used by the drop-in parity tests)."""
    if not DRIVER_SRC.exists():
        return None
    exe = LIBDIR / "tiled_driver"
    hdr = INCLUDE / "tiled_groupby_agg_partition.hpp"
    if not _stale(exe, [DRIVER_SRC, hdr, lib]):
        return exe
    cmd = [nvcc(), *ARCH, "-O2", "-std=c++17", "-I", str(INCLUDE), str(DRIVER_SRC), "-o", str(exe),
           "-L", str(LIBDIR), "-lgba", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    return exe


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
