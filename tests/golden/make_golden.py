"""Regenerate tests/golden/reference_tables.npz from the reference's own code.

Builds oracle/_ref/ref_tables with oracle/build_ref.sh (the reference's
TableKernel, BSpline/Wendland C4 kernels, Dim<3> geometry and
mapPositionThroughPlanes compiled unmodified from the reference source tree
against the stand-in Eigen/boost headers in oracle/refshim), runs it and packs
its raw outputs into one .npz.  Needs the reference tree, so it runs in the
development container only; the committed .npz is what the tests read.

    python tests/golden/make_golden.py
"""
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))


def main():
    exe = subprocess.check_output(["sh", os.path.join(ROOT, "oracle", "build_ref.sh")]).decode().strip().splitlines()[-1]
    with tempfile.TemporaryDirectory() as td:
        subprocess.check_call([exe, td])
        data = {}
        for f in sorted(os.listdir(td)):
            if f.endswith(".f64"):
                data[f[:-4]] = np.fromfile(os.path.join(td, f), dtype="<f8")
    out = os.path.join(HERE, "reference_tables.npz")
    np.savez_compressed(out, **data)
    print(out, sorted(data))


if __name__ == "__main__":
    main()
