"""The drop-in adapter inside the reference's own driver.

oracle/_ref/ref_sph_gpu is the reference's SPH path (FluidNodeList,
NestedGridNeighbor, ConnectivityMap, PeriodicBoundary, DataBase, State and
its policies, CheapSynchronousRK2, compiled from the reference's sources)
with llnl-spheral_b200/spheral/GpuSPHHydroBase.hh in place of SPHHydroBase:
the reference's integrator calls the adapter's evaluateDerivatives, which runs
on the GPU through libsphgpu.so.  On the committed SPH fixtures (what the
unmodified reference computed on the same inputs) the adapter's run must give:
  - every derivative field of the evaluation at the start time bit for bit,
    except the two that go through the ideal-H cube root (CUDA pow), within
    1e-12 normwise;
  - the hydro time-step vote and the state after the RK2 steps within 1e-12.
The binary is built where the reference tree is (oracle/build_ref.py); the
test is skipped without it."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, normwise
from test_oracle_reference import CASES, Fixture

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "oracle", "_ref", "ref_sph_gpu")
SPH_CASES = [c for c in CASES if not c.startswith("crk")]
POW_KEYS = {"weighted neighbor sum", "new H"}
STATE_KEYS = ["position", "velocity", "mass density", "specific thermal energy", "H", "pressure", "sound speed"]


def run_adapter(fx):
    """Run ref_sph_gpu on the fixture's input; its dumps by name."""
    with tempfile.TemporaryDirectory() as td:
        for sub in ("eval", "steps"):
            os.makedirs(os.path.join(td, sub))
        path = os.path.join(td, "in.bin")
        ns = fx.nodes
        with open(path, "wb") as f:
            f.write(np.int64(ns.n).tobytes())
            f.write(np.int64(fx.nsteps).tobytes())
            f.write(bytes(fx.cfg))
            for a in (ns.pos, ns.vel, ns.mass, ns.rho, ns.eps, ns.H):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        subprocess.run([EXE, path, td], check=True, stdout=subprocess.DEVNULL, timeout=600)
        out = {}
        for sub in ("eval", "steps"):
            d = os.path.join(td, sub)
            for name in os.listdir(d):
                if name.endswith(".f64"):
                    out[sub + "/" + name[:-4]] = np.fromfile(os.path.join(d, name), dtype="<f8")
    return out


@pytest.mark.skipif(not os.path.exists(EXE), reason="ref_sph_gpu is built where the reference tree is")
@pytest.mark.parametrize("name", SPH_CASES)
def test_adapter_in_the_reference_driver(gpu_lib, pkg, name):
    fx = Fixture(pkg, name)
    got = run_adapter(fx)
    for key in fx.eval_keys():
        a, b = got["eval/" + key], fx["eval/" + key]
        assert normwise(a, b) <= 1e-12, key
        if key not in POW_KEYS:
            assert np.array_equal(a, b), key
    dt, dtr = got["eval/hydro dt"][0], fx["eval/hydro dt"][0]
    assert abs(dt - dtr) <= 1e-12 * dtr
    assert normwise(got["steps/time_dt"], fx["steps/time_dt"]) <= 1e-12
    for key in STATE_KEYS:
        assert normwise(got["steps/" + key], fx["steps/" + key]) <= 1e-12, key
