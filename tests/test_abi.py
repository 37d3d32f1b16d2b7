"""The C-ABI library builds for sm_100a, loads, and exports every symbol that
include/*.h declares (no device call is made here)."""
import ctypes
import glob
import importlib
import os
import re
import shutil
import subprocess

import pytest

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


def test_config_struct_layout_matches_header(tmp_path):
    """The ctypes mirror has the C struct's size and every field's offset
    (the C side measured by compiling the header with the host compiler)."""
    abi = importlib.import_module("llnl-spheral_b200.abi")
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    names = [f[0] for f in abi.SphConfig._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "sphgpu.h"\nint main(void) {\n'
                   '  printf("%zu\\n", sizeof(sphgpu_config));\n' +
                   "".join('  printf("%%zu\\n", offsetof(sphgpu_config, %s));\n' % n for n in names) +
                   "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.check_call([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    assert ctypes.sizeof(abi.SphConfig) == out[0]
    for name, off in zip(names, out[1:]):
        assert getattr(abi.SphConfig, name).offset == off, name


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
