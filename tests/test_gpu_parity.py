"""GPU (CUDA sm_100a, through the C-ABI) against the CPU oracle.

Tolerances:
  - ghost sets and ConnectivityMap CSR: bit-exact (integer work);
  - plain FP64 derivatives: within 1e-12 normwise (||gpu - oracle||_inf /
    ||oracle||_inf), the tolerance of the hot-path specification.  The thread-
    per-node gather reproduces the reference's accumulation order, so all
    fields except the cube root of the ideal-H zeroth moment (CUDA pow vs
    glibc pow, <= 2 ulp) are in fact bit-exact, which is asserted too;
  - states after RK2 steps: 1e-12 normwise.
"""
import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu

DERIV_KEYS = ["delta velocity hydro", "delta specific thermal energy", "delta mass density", "delta position",
              "new mass density", "normalization", "velocity gradient", "internal velocity gradient",
              "M SPH gradient correction", "local M SPH gradient correction", "delta H", "new H",
              "weighted neighbor sum", "mass second moment", "max viscous pressure",
              "effective viscous pressure", "viscous work rate", "XSPH weight sum", "XSPH delta vi"]
POW_KEYS = {"weighted neighbor sum", "new H"}
STATE_KEYS = ["position", "velocity", "mass density", "specific thermal energy", "H", "pressure", "sound speed"]


def _sod(gen, abi, nx=32, ny=8, nz=8, **cfgkw):
    box = ((0.0, 0.0, 0.0), (1.0, ny / nx, nz / nx))
    ns = gen.sod(nx=nx, ny=ny, nz=nz, box=box)
    return ns, gen.sod_config(abi, ns_box=box, **cfgkw)


def _kh(gen, abi, nx=24, ny=24, nz=12, **cfgkw):
    ns = gen.kelvin_helmholtz(nx=nx, ny=ny, nz=nz, box=((0, 0, 0), (1.0, 1.0, nz / nx)))
    return ns, gen.kh_config(abi, xmax=(1.0, 1.0, nz / nx), **cfgkw)


CASES = {
    "sod": lambda g, a: _sod(g, a),
    "kh": lambda g, a: _kh(g, a),
    "sod_gradh_xsph": lambda g, a: _sod(g, a, gradhCorrection=1, XSPH=1),
    "sod_tensile_integrateH": lambda g, a: _sod(g, a, epsTensile=0.3, HUpdate=a.H_INTEGRATE),
    "kh_noncompatible_integrate_density": lambda g, a: _kh(g, a, compatibleEnergyEvolution=0,
                                                          densityUpdate=a.DENSITY_INTEGRATE),
    "sod_expansion_viscosity": lambda g, a: _sod(g, a, linearInExpansion=1, quadraticInExpansion=1, Cq=1.5),
    "sod_x_periodic_only": lambda g, a: _sod(g, a, periodic=(1, 0, 0)),
}


def _pair(pkg, oracle_mod, case):
    gen, abi = pkg.generators, pkg.abi
    ns, cfg = CASES[case](gen, abi)
    return pkg.SPHHydro(cfg, ns), oracle_mod.OracleProblem(cfg, ns), ns


@pytest.mark.parametrize("case", list(CASES))
def test_connectivity_bitexact(gpu_lib, pkg, oracle_mod, case):
    g, o, ns = _pair(pkg, oracle_mod, case)
    g.build_neighbors()
    o.build_neighbors()
    go, gn, gr = g.connectivity()
    oo, on, orr = o.connectivity()
    assert np.array_equal(gr, orr)
    assert np.array_equal(go, oo)
    assert np.array_equal(gn, on)
    assert g.num_pairs() == o.num_pairs()


@pytest.mark.parametrize("case", ["sod", "kh", "sod_x_periodic_only"])
@pytest.mark.parametrize("schedule", [1, 2])
@pytest.mark.parametrize("nfilter", [0, 1])
@pytest.mark.parametrize("passes", [1, 2])
@pytest.mark.parametrize("cells", [1, 2])
def test_connectivity_every_schedule(gpu_lib, pkg, oracle_mod, case, schedule, nfilter, passes, cells):
    """Thread-per-node and warp-per-node neighbor walks, with and without the
    FP32 pre-test, in one pass (lists parked in the pair-acceleration buffer,
    then compacted) or two (count, then fill), over cells of one kernel reach
    (27-cell window) or half a reach (125-cell window with distance pruning),
    give the same CSR."""
    g, o, ns = _pair(pkg, oracle_mod, case)
    g.set_schedule("neighbor walk", schedule)
    g.set_schedule("neighbor filter", nfilter)
    g.set_schedule("neighbor passes", passes)
    g.set_schedule("neighbor cells", cells)
    g.build_neighbors()
    assert g.schedule("neighbor walk") == schedule
    assert g.schedule("neighbor passes") == passes
    assert g.schedule("neighbor cells") == cells
    o.build_neighbors()
    go, gn, gr = g.connectivity()
    oo, on, orr = o.connectivity()
    assert np.array_equal(go, oo)
    assert np.array_equal(gn, on)
    assert g.num_pairs() == o.num_pairs()


@pytest.mark.parametrize("case", ["sod", "kh", "sod_x_periodic_only"])
@pytest.mark.parametrize("passes", [1, 2])
def test_ghost_passes_every_schedule(gpu_lib, pkg, oracle_mod, case, passes):
    """The six boundary passes as four launches and a prefix sum each, or all
    in one cooperative launch with grid barriers, make the reference's ghosts
    (roots, positions, order) and the same CSR."""
    g, o, ns = _pair(pkg, oracle_mod, case)
    g.set_schedule("ghost passes", passes)
    g.build_neighbors()
    assert g.schedule("ghost passes") == passes
    o.build_neighbors()
    go, gn, gr = g.connectivity()
    oo, on, orr = o.connectivity()
    assert np.array_equal(gr, orr)
    assert np.array_equal(g.ghost_positions(), o.ghost_positions())
    assert np.array_equal(go, oo)
    assert np.array_equal(gn, on)
    # and again after steps (the graph-replayed rebuild)
    g.step(3)
    o.step(3)
    assert np.array_equal(g.connectivity()[2], o.connectivity()[2])
    assert np.array_equal(g.connectivity()[1], o.connectivity()[1])


@pytest.mark.parametrize("case", list(CASES))
def test_evaluate_derivatives_parity(gpu_lib, pkg, oracle_mod, case):
    g, o, ns = _pair(pkg, oracle_mod, case)
    g.build_neighbors()
    o.build_neighbors()
    g.initialize()
    o.initialize()
    g.evaluateDerivatives()
    o.evaluate_derivatives()
    for k in DERIV_KEYS:
        a, b = g.field(k), o.field(k)
        assert normwise(a, b) <= 1e-12, k
        if k not in POW_KEYS:
            assert np.array_equal(a, b), k
    assert g.dt() == o.dt()


@pytest.mark.parametrize("case", ["sod", "kh", "sod_gradh_xsph", "sod_tensile_integrateH",
                                  "kh_noncompatible_integrate_density"])
def test_rk2_steps_parity(gpu_lib, pkg, oracle_mod, case):
    g, o, ns = _pair(pkg, oracle_mod, case)
    g.build_neighbors()
    o.build_neighbors()
    g.evaluateDerivatives()
    o.evaluate_derivatives()
    for _ in range(8):
        tg, dtg = g.step(1)
        to, dto = o.step(1)
        assert abs(dtg - dto) <= 1e-12 * dto
    for k in STATE_KEYS:
        assert normwise(g.field(k), o.field(k)) <= 1e-12, k
    for k in ("delta velocity hydro", "delta specific thermal energy", "delta mass density"):
        assert normwise(g.field(k), o.field(k)) <= 1e-12, k


def test_energy_conservation_compatible(gpu_lib, pkg):
    gen, abi = pkg.generators, pkg.abi
    ns, cfg = _sod(gen, abi, nx=64, ny=8, nz=8)
    g = pkg.SPHHydro(cfg, ns)
    g.build_neighbors()
    g.evaluateDerivatives()
    c0 = g.conservation()
    g.step(20)
    c1 = g.conservation()
    assert abs(c1[6] - c0[6]) <= 1e-12 * abs(c0[6])
    assert np.all(np.abs(c1[1:4]) <= 1e-12 * c0[0])


@pytest.mark.parametrize("shrink", [5.0, 1.6])
def test_sparse_and_empty_neighbor_lists(gpu_lib, pkg, oracle_mod, shrink):
    """shrink 5: kappa*h < node spacing, so every list is empty (E = 0) and the
    zero-neighbor branches run (M not inverted, Wsum = 0 ideal H, omega = 1);
    shrink 1.6: ragged lists of a few neighbors each."""
    gen, abi = pkg.generators, pkg.abi
    ns, cfg = _sod(gen, abi, nx=16, ny=4, nz=4, gradhCorrection=1)
    ns.H[:, [0, 3, 5]] *= shrink
    g = pkg.SPHHydro(cfg, ns)
    o = oracle_mod.OracleProblem(cfg, ns)
    g.build_neighbors()
    o.build_neighbors()
    go, gn, _ = g.connectivity()
    oo, on, _ = o.connectivity()
    assert np.array_equal(go, oo) and np.array_equal(gn, on)
    if shrink == 5.0:
        assert len(gn) == 0
    g.initialize()
    o.initialize()
    g.evaluateDerivatives()
    o.evaluate_derivatives()
    for k in DERIV_KEYS + ["grad h corrections"]:
        assert normwise(g.field(k), o.field(k)) <= 1e-12, k


def test_error_paths_return_status(gpu_lib, pkg):
    gen, abi = pkg.generators, pkg.abi
    ns, cfg = _sod(gen, abi, nx=16, ny=4, nz=4)
    g = pkg.SPHHydro(cfg, n=ns.n)
    with pytest.raises(RuntimeError, match="connectivity not built"):
        g.evaluateDerivatives()
    bad = gen.NodeSet(ns.pos, ns.vel, -ns.mass, ns.rho, ns.eps, ns.H, ns.dx)
    with pytest.raises(RuntimeError, match="non-positive"):
        g.set_state(bad)
    # more neighbors than the per-node capacity is reported, not truncated
    cfg2 = cfg.copy()
    cfg2.max_neighbors = 64
    g2 = pkg.SPHHydro(cfg2, ns)
    with pytest.raises(RuntimeError, match="neighbor"):
        g2.build_neighbors()
    # the same problem still works after the error
    g.set_state(ns)
    g.build_neighbors()
    g.evaluateDerivatives()


def test_large_neighbor_counts(gpu_lib, pkg, oracle_mod):
    """nPerh = 3 gives ~900 neighbors per node with the B-spline (capacity 1024)."""
    gen, abi = pkg.generators, pkg.abi
    ns, cfg = _sod(gen, abi, nx=24, ny=8, nz=8, nPerh=3.0)
    ns.H[:, [0, 3, 5]] = 1.0 / (3.0 * ns.dx[0])
    g = pkg.SPHHydro(cfg, ns)
    o = oracle_mod.OracleProblem(cfg, ns)
    g.build_neighbors()
    o.build_neighbors()
    go, gn, _ = g.connectivity()
    oo, on, _ = o.connectivity()
    assert np.array_equal(gn, on) and np.array_equal(go, oo)
    assert np.diff(go).max() > 700
    g.evaluateDerivatives()
    o.evaluate_derivatives()
    assert np.array_equal(g.field("delta velocity hydro"), o.field("delta velocity hydro"))


def test_single_pass_needs_the_pair_acceleration_buffer(gpu_lib, pkg, oracle_mod):
    """Without compatible energy there is no pair-acceleration buffer to park
    the lists in: the build counts, then fills, with the same CSR."""
    g, o, ns = _pair(pkg, oracle_mod, "kh_noncompatible_integrate_density")
    g.build_neighbors()
    o.build_neighbors()
    assert g.schedule("neighbor passes") == 2
    go, gn, _ = g.connectivity()
    oo, on, _ = o.connectivity()
    assert np.array_equal(go, oo) and np.array_equal(gn, on)
    k, ok, _ = _pair(pkg, oracle_mod, "kh")
    k.build_neighbors()
    assert k.schedule("neighbor passes") == 1


def test_empty_problem_rejected(gpu_lib, pkg):
    abi = pkg.abi
    import ctypes
    h = ctypes.c_void_p()
    cfg = abi.make_config()
    assert gpu_lib.sphgpu_create(ctypes.byref(cfg), 0, ctypes.byref(h)) == abi.ERR_ARG


@pytest.mark.parametrize("nfilter", [0, 1])
@pytest.mark.parametrize("cells", [1, 2])
def test_connectivity_anisotropic_h(gpu_lib, pkg, oracle_mod, nfilter, cells):
    """Anisotropic, varied H (condition numbers up to ~2) with the eta_i OR
    eta_j predicate: many candidates sit near the support boundary."""
    gen, abi = pkg.generators, pkg.abi
    box = ((0.0, 0.0, 0.0), (1.0, 0.25, 0.25))
    ns = gen.sod(nx=32, ny=8, nz=8, box=box, jitter=0.2, seed=5)
    rng = np.random.default_rng(9)
    ns.H[:, 0] *= rng.uniform(0.7, 1.4, ns.n)
    ns.H[:, 3] *= rng.uniform(0.7, 1.4, ns.n)
    ns.H[:, 5] *= rng.uniform(0.7, 1.4, ns.n)
    ns.H[:, 1] = 0.1 * ns.H[:, 0] * rng.uniform(-1, 1, ns.n)
    ns.H[:, 4] = 0.1 * ns.H[:, 3] * rng.uniform(-1, 1, ns.n)
    cfg = gen.sod_config(abi, ns_box=box)
    g = pkg.SPHHydro(cfg, ns)
    g.set_schedule("neighbor filter", nfilter)
    g.set_schedule("neighbor cells", cells)
    o = oracle_mod.OracleProblem(cfg, ns)
    g.build_neighbors()
    o.build_neighbors()
    go, gn, gr = g.connectivity()
    oo, on, orr = o.connectivity()
    assert np.array_equal(go, oo) and np.array_equal(gn, on) and np.array_equal(gr, orr)


@pytest.mark.parametrize("case", ["sod", "kh"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pair_accelerations_reference_layout(gpu_lib, pkg, oracle_mod, case, precision):
    """sphgpu_get_pair_accelerations against the oracle's pair-wise
    accelerations (the reference's layout, bit-pinned to the reference): the
    entries of the pairs a node owns (neighbor j > i or a ghost) are
    bit-identical in FP64; the others (m_owner deltaDvDt formed from the
    owner's value) agree to rounding.  Before an evaluation on the current
    connectivity there are none to read."""
    g, o, ns = _pair(pkg, oracle_mod, case)
    g.build_neighbors()
    with pytest.raises(RuntimeError):
        g.pair_accelerations()
    if precision == "mixed":
        gen, abi = pkg.generators, pkg.abi
        ns2, cfg2 = CASES[case](gen, abi)
        cfg2.precision = abi.PRECISION_MIXED
        g = pkg.SPHHydro(cfg2, ns2)
        g.build_neighbors()
    g.evaluateDerivatives()
    o.build_neighbors()
    o.evaluate_derivatives()
    off, nb, _ = g.connectivity()
    row = np.repeat(np.arange(ns.n), np.diff(off))
    own = nb > row
    a, b = g.pair_accelerations(), o.pair_accelerations()
    assert a.shape == b.shape
    scale = np.max(np.abs(b))
    if precision == "fp64":
        assert np.array_equal(a[own], b[own])
        assert np.max(np.abs(a[~own] - b[~own])) <= 1e-14 * scale
    else:
        assert np.max(np.abs(a - b)) <= 1e-5 * scale


def _canonical(h, n, L):
    """Rows as sorted lists of (node, periodic image) of the current connectivity."""
    off, nb, root = h.connectivity()
    gpos = h.ghost_positions()
    pos = h.field("position")
    rows = []
    for i in range(n):
        row = []
        for j in nb[off[i]:off[i + 1]]:
            if j < n:
                row.append((int(j), 0, 0, 0))
            else:
                r = int(root[j - n])
                s = np.rint((gpos[j - n] - pos[r]) / L).astype(int)
                row.append((r, int(s[0]), int(s[1]), int(s[2])))
        rows.append(row)
    return rows


@pytest.mark.parametrize("case", ["sod", "kh"])
def test_shuffled_input_order(gpu_lib, pkg, case):
    """The caller's node order is arbitrary (the reference numbers nodes as
    the generator lays them out, but nothing depends on it): a seeded
    permutation of the input gives the same neighbor sets after mapping the
    indices back, each row still ascending in the caller's numbering, the
    same pair count, and derivatives equal within 1e-12 (the rows visit the
    pairs in another order, so the sums round differently)."""
    gen, abi = pkg.generators, pkg.abi
    ns, cfg = CASES[case](gen, abi)
    perm = np.random.default_rng(11).permutation(ns.n)
    sh = gen.NodeSet(ns.pos[perm], ns.vel[perm], ns.mass[perm], ns.rho[perm], ns.eps[perm], ns.H[perm], ns.dx)
    g, gs = pkg.SPHHydro(cfg, ns), pkg.SPHHydro(cfg, sh)
    g.build_neighbors()
    gs.build_neighbors()
    assert g.num_pairs() == gs.num_pairs()
    L = np.array(cfg.xmax) - np.array(cfg.xmin)
    rows, rows_s = _canonical(g, ns.n, L), _canonical(gs, ns.n, L)
    off, nb, _ = gs.connectivity()
    for k in range(ns.n):
        internal = nb[off[k]:off[k + 1]]
        internal = internal[internal < ns.n]
        assert np.all(np.diff(internal) > 0)
        mapped = sorted((int(perm[a]), sx, sy, sz) for a, sx, sy, sz in rows_s[k])
        assert mapped == sorted(rows[perm[k]])
    g.evaluateDerivatives()
    gs.evaluateDerivatives()
    inv = np.argsort(perm)
    for key in ("delta velocity hydro", "delta specific thermal energy", "velocity gradient", "new mass density"):
        a = g.field(key).reshape(ns.n, -1)
        b = gs.field(key).reshape(ns.n, -1)[inv]
        assert normwise(b.ravel(), a.ravel()) <= 1e-12, key
