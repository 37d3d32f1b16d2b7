"""The CUDA path against the reference's own SPH / CRKSPH path, executed.

Same fixtures as tests/test_oracle_reference.py (what the reference's
SPHHydroBase / CRKSPHHydroBase, ConnectivityMap, PeriodicBoundary and
CheapSynchronousRK2, compiled from its sources, computed on small seeded node
sets), read through the C-ABI.  Tolerances:
  - ghosts and ConnectivityMap: bit-exact, neighbors compared as (root node,
    ghost position) in row order (the reference culls unused ghosts, which
    renumbers them but keeps the order);
  - derivatives of one evaluateDerivatives: bit-exact, except the fields
    that go through the cube root of the ideal-H zeroth moment (CUDA pow vs
    glibc pow, <= 2 ulp) and, with the CRKSPH Q, its limiter's exp: within
    1e-12 normwise (||gpu - ref||_inf / ||ref||_inf), the tolerance of the
    hot-path specification;
  - the hydro time-step vote: equal;
  - the state after the RK2 steps: within 1e-12 normwise.
"""
import numpy as np
import pytest

from conftest import normwise
from test_oracle_reference import CASES, Fixture, canonical_rows

pytestmark = pytest.mark.gpu

POW_KEYS = {"weighted neighbor sum", "new H"}
STATE_KEYS = ["position", "velocity", "mass density", "specific thermal energy", "H", "pressure", "sound speed"]


@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_reference(gpu_lib, pkg, name):
    fx = Fixture(pkg, name)
    g = pkg.SPHHydro(fx.cfg, fx.nodes)
    g.build_neighbors()
    off, nb, root = g.connectivity()
    assert canonical_rows(fx.n, off, nb, root, g.ghost_positions()) == fx.rows()
    g.initialize()
    g.evaluateDerivatives()
    exp_q = fx.cfg.qType == pkg.abi.Q_CRKSPH_MONAGHAN_GINGOLD
    for key in fx.eval_keys():
        a, b = g.field(key).ravel(), fx["eval/" + key]
        assert normwise(a, b) <= 1e-12, key
        if key not in POW_KEYS and not exp_q:
            assert np.array_equal(a, b), key
    dt = g.dt()
    assert abs(dt - fx["eval/hydro dt"][0]) <= 1e-12 * fx["eval/hydro dt"][0]
    if not exp_q:
        assert dt == fx["eval/hydro dt"][0]
    t, last = g.step(fx.nsteps)
    tr, dtr = fx["steps/time_dt"][-2:]
    assert abs(t - tr) <= 1e-12 * tr and abs(last - dtr) <= 1e-12 * dtr
    for key in STATE_KEYS:
        assert normwise(g.field(key).ravel(), fx["steps/" + key]) <= 1e-12, key
    if fx.cfg.hydro == pkg.abi.HYDRO_CRKSPH:
        assert normwise(g.field("node volume").ravel(), fx["steps/node volume"]) <= 1e-12


from test_oracle_reference import IDEALH, idealh_fixture  # noqa: E402


@pytest.mark.parametrize("path", IDEALH, ids=[p.split("/")[-1][:-4] for p in IDEALH])
def test_gpu_iterate_ideal_h_matches_reference(gpu_lib, pkg, path):
    """sphgpu_iterate_ideal_h against the reference's iterateIdealH: same
    iteration count, the last change to the reference's printed digits, H
    within 1e-12 (the cube root of the zeroth moment is CUDA's pow)."""
    d, cfg, nodes = idealh_fixture(pkg, path)
    g = pkg.SPHHydro(cfg, nodes)
    itr, dh = g.iterateIdealH(int(d["input/max_iterations"]), float(d["input/tolerance"]))
    assert itr == int(d["iterations"])
    assert abs(dh - float(d["max_delta_h_printed"])) <= 1e-5 * dh
    assert normwise(g.field("H").ravel(), d["H"]) <= 1e-12
