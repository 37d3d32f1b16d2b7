"""Mixed-precision form (FP32 pair arithmetic, Kahan FP32 sums, FP64 state)
against the plain FP64 GPU path and the oracle.

Tolerances (from the hot-path specification): every derivative field within
1e-5 max relative error, normwise (||mixed - fp64||_inf / ||fp64||_inf);
relative total-energy drift <= 1e-6 over 200 RK2 steps.
"""
import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu

FIELDS = ["delta velocity hydro", "delta specific thermal energy", "delta mass density", "velocity gradient",
          "new mass density", "new H", "M SPH gradient correction", "max viscous pressure"]


def _evolved_sod(pkg, steps=5):
    gen, abi = pkg.generators, pkg.abi
    box = ((0.0, 0.0, 0.0), (1.0, 0.125, 0.125))
    ns = gen.sod(nx=64, ny=8, nz=8, box=box)
    cfg = gen.sod_config(abi, ns_box=box)
    g = pkg.SPHHydro(cfg, ns)
    g.build_neighbors()
    g.evaluateDerivatives()
    g.step(steps)
    pos, vel, rho, eps, H = (g.field(k) for k in ("position", "velocity", "mass density",
                                                  "specific thermal energy", "H"))
    return gen.NodeSet(pos, vel, ns.mass, rho, eps, H, ns.dx), cfg


@pytest.mark.parametrize("which", ["sod_evolved", "kh"])
def test_mixed_derivative_errors(gpu_lib, pkg, oracle_mod, which):
    gen, abi = pkg.generators, pkg.abi
    if which == "sod_evolved":
        ns, cfg = _evolved_sod(pkg)
    else:
        ns = gen.kelvin_helmholtz(nx=32, ny=32, nz=16, box=((0, 0, 0), (1.0, 1.0, 0.5)))
        cfg = gen.kh_config(abi, xmax=(1.0, 1.0, 0.5))
    cm = cfg.copy()
    cm.precision = abi.PRECISION_MIXED
    f = pkg.SPHHydro(cfg, ns)
    m = pkg.SPHHydro(cm, ns)
    o = oracle_mod.OracleProblem(cfg, ns)
    for p in (f, m):
        p.build_neighbors()
        p.evaluateDerivatives()
    o.build_neighbors()
    o.evaluate_derivatives()
    for k in FIELDS:
        ref = o.field(k)
        assert normwise(f.field(k), ref) <= 1e-12, k
        assert normwise(m.field(k), ref) <= 1e-5, k


def test_mixed_energy_drift_200_steps(gpu_lib, pkg):
    gen, abi = pkg.generators, pkg.abi
    box = ((0.0, 0.0, 0.0), (1.0, 0.125, 0.125))
    ns = gen.sod(nx=64, ny=8, nz=8, box=box)
    cfg = gen.sod_config(abi, ns_box=box, precision=abi.PRECISION_MIXED)
    m = pkg.SPHHydro(cfg, ns)
    m.build_neighbors()
    m.evaluateDerivatives()
    e0 = m.conservation()[6]
    m.step(200)
    e1 = m.conservation()[6]
    assert abs(e1 - e0) / abs(e0) <= 1e-6


@pytest.mark.parametrize("which", ["sod", "kh"])
def test_mixed_summed_density_and_states_after_steps(gpu_lib, pkg, which):
    """The mixed form also sums the density (RigorousSumDensity) with FP32
    pair terms and a Kahan sum: after a few RK2 steps the states stay within
    1e-5 of the FP64 path, and finalize() alone gives the density within it."""
    gen, abi = pkg.generators, pkg.abi
    if which == "sod":
        box = ((0.0, 0.0, 0.0), (1.0, 0.125, 0.125))
        ns = gen.sod(nx=64, ny=8, nz=8, box=box)
        cfg = gen.sod_config(abi, ns_box=box)
    else:
        ns = gen.kelvin_helmholtz(nx=32, ny=32, nz=16, box=((0, 0, 0), (1.0, 1.0, 0.5)))
        cfg = gen.kh_config(abi, xmax=(1.0, 1.0, 0.5))
    cm = cfg.copy()
    cm.precision = abi.PRECISION_MIXED
    f = pkg.SPHHydro(cfg, ns)
    m = pkg.SPHHydro(cm, ns)
    for p in (f, m):
        p.build_neighbors()
        p.finalize()
    assert normwise(m.field("mass density"), f.field("mass density")) <= 1e-6
    for p in (f, m):
        p.step(5)
    for k in ("mass density", "position", "velocity", "specific thermal energy", "H"):
        assert normwise(m.field(k), f.field(k)) <= 1e-5, k


def test_mixed_balsara_after_steps(gpu_lib, pkg, oracle_mod):
    """The Balsara shear correction in both forms: after 3 RK2 steps (the
    correction is zero at the first evaluation, where the velocity gradient
    of a previous one is zero) the FP64 state is within 1e-12 of the oracle's
    and the mixed form's within 1e-5; a CRKSPH problem with the correction
    is refused."""
    gen, abi = pkg.generators, pkg.abi
    ns = gen.kelvin_helmholtz(nx=24, ny=24, nz=12, box=((0, 0, 0), (1.0, 1.0, 0.5)))
    cfg = gen.kh_config(abi, xmax=(1.0, 1.0, 0.5), balsaraShearCorrection=1)
    cm = cfg.copy()
    cm.precision = abi.PRECISION_MIXED
    f, m, o = pkg.SPHHydro(cfg, ns), pkg.SPHHydro(cm, ns), oracle_mod.OracleProblem(cfg, ns)
    for p in (f, m):
        p.build_neighbors()
        p.evaluateDerivatives()
        p.step(3)
    o.build_neighbors()
    o.evaluate_derivatives()
    o.step(3)
    for k in ("velocity", "specific thermal energy", "mass density", "H"):
        ref = o.field(k)
        assert normwise(f.field(k), ref) <= 1e-12, k
        assert normwise(m.field(k), ref) <= 1e-5, k
    f.build_neighbors()
    o.build_neighbors()
    f.initialize()
    o.initialize()
    f.evaluateDerivatives()
    o.evaluate_derivatives()
    assert normwise(f.field("max viscous pressure"), o.field("max viscous pressure")) <= 1e-12
    assert np.max(o.field("max viscous pressure")) > 0.0
    with pytest.raises(RuntimeError):
        pkg.SPHHydro(gen.kh_config(abi, xmax=(1.0, 1.0, 0.5), hydro=abi.HYDRO_CRKSPH, balsaraShearCorrection=1), ns)
