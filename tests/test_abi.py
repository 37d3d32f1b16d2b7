"""The C-ABI library builds for sm_100a, loads, and exports every symbol that
include/*.h declares (no device call is made here)."""
import ctypes
import glob
import importlib
import os
import re

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(sphgpu_[A-Za-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("sphgpu_create", "sphgpu_evaluate_derivatives", "sphgpu_step_rk2", "sphgpu_build_neighbors",
                 "sphgpu_get_connectivity", "sphgpu_finalize", "sphgpu_dt", "sphgpu_last_error"):
        assert must in names


def test_library_exports_all_declared_symbols():
    build = importlib.import_module("llnl-spheral_b200.build")
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_config_struct_layout_matches_header():
    abi = importlib.import_module("llnl-spheral_b200.abi")
    # 4 ints, 1 double, 3 doubles, 2 ints, 1 + 2 + 3 + 2 + 1 doubles, 8 ints,
    # 6 doubles, 4 ints, 4 doubles
    expect = 4 * 4 + 8 + 24 + 8 + 8 + 16 + 24 + 16 + 8 + 32 + 48 + 16 + 32
    assert ctypes.sizeof(abi.SphConfig) == expect


def test_error_codes_without_gpu_calls():
    abi = importlib.import_module("llnl-spheral_b200.abi")
    lib = abi.load_library()
    comps = ctypes.c_int32()
    assert lib.sphgpu_field_components(b"delta velocity hydro", ctypes.byref(comps)) == abi.OK
    assert comps.value == 3
    assert lib.sphgpu_field_components(b"no such field", ctypes.byref(comps)) == abi.ERR_ARG
    assert b"unknown field key" in lib.sphgpu_last_error()
    # bad arguments are rejected before any device work
    h = ctypes.c_void_p()
    assert lib.sphgpu_create(None, 10, ctypes.byref(h)) == abi.ERR_ARG
    cfg = abi.make_config(num_points=2)
    assert lib.sphgpu_create(ctypes.byref(cfg), 10, ctypes.byref(h)) == abi.ERR_ARG
    cfg = abi.make_config(hydro=7)
    assert lib.sphgpu_create(ctypes.byref(cfg), 10, ctypes.byref(h)) in (abi.ERR_ARG, abi.ERR_UNSUPPORTED)
