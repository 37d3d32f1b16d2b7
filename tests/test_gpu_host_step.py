"""sphgpu_step_rk2_host: one CheapSynchronousRK2 step of a state held in host
arrays (src/Integrator/CheapSynchronousRK2.cc:81-143 with the reference's
Fields on the host) gives, bit for bit, what sphgpu_set_state +
sphgpu_step_rk2 + sphgpu_get_state give, step after step, for SPH (whose
rebuild overlaps the copies of the rest of the state) and CRKSPH."""
import ctypes
from types import SimpleNamespace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "mass", "rho", "eps", "H")


def _case(pkg, which):
    gen, abi = pkg.generators, pkg.abi
    if which.startswith("sod"):
        box = ((0.0, 0.0, 0.0), (1.0, 0.25, 0.25))
        ns = gen.sod(nx=32, ny=8, nz=8, box=box)
        cfg = gen.sod_config(abi, ns_box=box)
    else:
        ns = gen.kelvin_helmholtz(nx=16, ny=16, nz=8, box=((0, 0, 0), (1.0, 1.0, 0.5)))
        cfg = gen.kh_config(abi, xmax=(1.0, 1.0, 0.5),
                            **({"hydro": abi.HYDRO_CRKSPH} if which.endswith("crk") else {}))
    if "mixed" in which:
        cfg.precision = abi.PRECISION_MIXED
    return ns, cfg


def _arrays(ns):
    return [np.ascontiguousarray(getattr(ns, k), dtype=np.float64).copy() for k in FIELDS]


@pytest.mark.parametrize("which", ["kh", "kh_mixed", "sod", "kh_crk"])
def test_host_step_equals_set_step_get(gpu_lib, pkg, which):
    ns, cfg = _case(pkg, which)
    a = _arrays(ns)           # state of the host-step run (in and out through the same arrays)
    b = _arrays(ns)           # state of the set_state / step_rk2 / get_state run
    ha = pkg.SPHHydro(cfg, n=ns.n)
    hb = pkg.SPHHydro(cfg, n=ns.n)
    for step in range(4):
        ta, dta = ha.step_host(a)
        hb.set_state(SimpleNamespace(**dict(zip(FIELDS, b))))
        tb, dtb = hb.step(1)
        out = [np.empty_like(x) for x in b]
        assert gpu_lib.sphgpu_get_state(hb.h, *[x.ctypes.data_as(ctypes.c_void_p) for x in out]) == 0
        b = out
        assert ta == tb and dta == dtb, step
        for k, x, y in zip(FIELDS, a, b):
            assert np.array_equal(x, y), (step, k)
    ha.close()
    hb.close()


def test_host_step_separate_and_skipped_outputs(gpu_lib, pkg):
    ns, cfg = _case(pkg, "kh")
    a = _arrays(ns)
    keep = [x.copy() for x in a]
    ha = pkg.SPHHydro(cfg, n=ns.n)
    out = [np.empty_like(x) for x in a]
    out[2] = None                      # mass not read back
    ha.step_host(a, out)
    for x, y in zip(a, keep):
        assert np.array_equal(x, y)    # inputs untouched
    hb = pkg.SPHHydro(cfg, ns)
    hb.step(1)
    for k, x in zip(("position", "velocity", None, "mass density", "specific thermal energy", "H"), out):
        if k is not None:
            assert np.array_equal(x, hb.field(k)), k
    ha.close()
    hb.close()


def test_host_step_requires_every_input(gpu_lib, pkg):
    ns, cfg = _case(pkg, "sod")
    a = _arrays(ns)
    h = pkg.SPHHydro(cfg, n=ns.n)
    ptrs = [x.ctypes.data_as(ctypes.c_void_p) for x in a]
    ptrs[3] = None
    t = ctypes.c_double(0.0)
    dt = ctypes.c_double()
    rc = gpu_lib.sphgpu_step_rk2_host(h.h, *ptrs, *ptrs, ctypes.byref(t), ctypes.byref(dt))
    assert rc == pkg.abi.ERR_ARG
    h.close()
