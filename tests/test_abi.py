"""The C ABI library loads and exports every symbol include/*.h declares (CPU only)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A

ROOT = Path(__file__).resolve().parents[1]


def _declared_functions(header: Path) -> set[str]:
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(gba_[a-z0-9_]+)\s*\(", text)) - {"gba_gen_spec"}


def test_library_exports_every_declared_function():
    lib = A.lib()
    declared = _declared_functions(ROOT / "include" / "gba.h")
    assert len(declared) >= 19
    missing = [f for f in declared if not hasattr(lib, f)]
    assert not missing, missing
    # and the binding covers every declared function
    assert declared == set(A.SIGNATURES), declared ^ set(A.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", str(A.LIB_PATH)], capture_output=True, text=True).stdout
    for f in declared:
        assert re.search(rf"\bT {f}\b", out), f


def test_struct_layouts_match_binding():
    lib = A.lib()
    for which, cls in enumerate([A.Query, A.Output, A.Knobs, A.Stats, A.GenSpec, A.ServerConfig, A.RequestInfo]):
        assert lib.gba_abi_struct_size(which) == C.sizeof(cls), cls.__name__


def test_default_knobs_and_status_strings():
    lib = A.lib()
    k = A.Knobs()
    lib.gba_default_knobs(C.byref(k))
    assert k.load_factor == 0.5 and k.preagg == -1 and k.max_regrow == 4
    for s in range(9):
        assert lib.gba_status_string(s)


def test_no_gpu_calls_fail_cleanly():
    """Without a usable device gba_create reports an error instead of crashing."""
    import torch
    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    assert A.lib().gba_create(C.byref(h), 0) != A.OK


def test_invalid_arguments_rejected_without_gpu():
    lib = A.lib()
    assert lib.gba_groupby(None, None, None, None, None, None) == A.ERR_INVALID_ARG
    assert lib.gba_destroy(None) == A.ERR_INVALID_ARG


def test_dropin_cxx_entry_points_exported():
    """The reference's C++ entry points (include/tiled_groupby_agg_partition.hpp)
    are defined in libgba.so, and the test.cu-style caller links against it."""
    out = subprocess.run(["nm", "-DC", "--defined-only", str(A.LIB_PATH)], capture_output=True, text=True).stdout
    assert "groupby_agg_partition<unsigned int, unsigned int>(unsigned int*, unsigned int*, unsigned long, " \
           "unsigned long, unsigned long, std::vector<par_result" in out
    assert "groupby_agg_intra_partition(std::vector<par_result" in out
    driver = A.LIB_PATH.parent / "tiled_driver"
    assert driver.exists()
    ldd = subprocess.run(["ldd", str(driver)], capture_output=True, text=True).stdout
    assert "libgba.so" in ldd and "not found" not in ldd.split("libgba.so")[1].splitlines()[0]


def test_c_caller_compiles_and_links(tmp_path):
    """include/gba.h is plain C11: a C caller using every struct field the
    guide shows compiles without warnings and links against libgba.so."""
    src = ROOT / "tests" / "drivers" / "c_caller.c"
    out = tmp_path / "c_caller.so"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Wno-missing-field-initializers", "-Werror",
                        "-I", str(ROOT / "include"), "-shared", "-fPIC", str(src), "-o", str(out),
                        "-L", str(A.LIB_PATH.parent), "-lgba"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
