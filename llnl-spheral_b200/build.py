"""Build libsphgpu.so (CUDA sm_100a kernels + C-ABI) in-tree with nvcc.

FP64 parity translation units are compiled with -fmad=false so that no FMA is
contracted: their per-pair arithmetic matches the x86-64 FP64 reference bit
for bit.  The mixed-precision units are too: otherwise the compiler may
contract the one-problem and the batched instances of a kernel differently,
and a batch member would differ from its solo run in the last bits.

    python llnl-spheral_b200/build.py [--force] [--verbose]
"""
import argparse
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libsphgpu.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I" + os.path.join(HERE, "..", "include")]
# (source, extra flags)
UNITS = [
    ("api.cu", ["-fmad=false"]),
    ("batch.cu", []),
    ("nbrs.cu", ["-fmad=false"]),
    ("sph.cu", ["-fmad=false"]),
    ("sph_mixed.cu", ["-fmad=false"]),
    ("crk.cu", ["-fmad=false"]),
    ("crk_mixed.cu", ["-fmad=false"]),
    ("noalloc.cu", []),
    ("server.cu", []),
    ("restart.cu", []),
    ("table.cc", []),
]
HEADERS = ["devmath.cuh", "problem.cuh", "mixed.cuh"]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = _mtime(LIB)
    deps = [os.path.join(CSRC, u) for u, _ in UNITS] + [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "sphgpu.h"))
    deps.append(os.path.abspath(__file__))
    return any(_mtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False, lib_path=None, extra_flags=()):
    """Compile every unit (in parallel) and link the library.  lib_path and
    extra_flags (e.g. -D tuning constants) build a variant elsewhere."""
    lib = lib_path or LIB
    if lib_path is None and not force and not needs_build():
        return LIB
    objdir = os.path.join(os.path.dirname(lib), "obj_" + os.path.basename(lib).replace(".", "_"))
    os.makedirs(objdir, exist_ok=True)
    cmds = []
    for src, extra in UNITS:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(objdir, src + ".o")
        cmd = [NVCC] + ARCH + COMMON + extra + list(extra_flags) + ["-c", path, "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if src.endswith(".cc"):
            cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off",
                   "-fno-fast-math", "-c", path, "-o", obj]
        cmds.append((cmd, obj))
    with concurrent.futures.ThreadPoolExecutor(min(len(cmds), os.cpu_count() or 4)) as ex:
        for cmd, r in zip(cmds, ex.map(lambda c: subprocess.run(c[0], capture_output=True, text=True), cmds)):
            if verbose or ptxas_info:
                print(" ".join(cmd[0]), flush=True)
                sys.stdout.write(r.stdout + r.stderr)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, cmd[0])
    cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + [o for _, o in cmds] + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info))
    sys.exit(0)
