"""Batched launches: a member of a batch gives exactly the results it gives alone.

Every stage of a batch call is one kernel launch over all members (a
per-member block map), and every member keeps its own buffers, so the
per-node arithmetic and its order are those of the member alone: states,
connectivity and dt are compared bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE_KEYS = ["position", "velocity", "mass density", "specific thermal energy", "H", "pressure", "sound speed"]


def _sod_member(pkg, nx, gamma, ratio, precision, seed):
    gen, abi = pkg.generators, pkg.abi
    k = max(4, nx // 8)
    box = ((0.0, 0.0, 0.0), (1.0, k / nx, k / nx))
    ns = gen.sod(nx=nx, ny=k, nz=k, box=box, gamma=gamma, rho1=1.0, rho2=1.0 / ratio, P1=1.0,
                 P2=0.1795, jitter=0.01, seed=seed)
    ns.vel[:, 0] = 0.02 * np.sin(2 * np.pi * ns.pos[:, 0])
    cfg = gen.sod_config(abi, ns_box=box, gamma=gamma, precision=precision)
    return ns, cfg


def _kh_member(pkg, precision, hydro=None):
    gen, abi = pkg.generators, pkg.abi
    ns = gen.kelvin_helmholtz(nx=16, ny=16, nz=8, box=((0, 0, 0), (1.0, 1.0, 0.5)))
    kw = dict(xmax=(1.0, 1.0, 0.5), precision=precision)
    if hydro is not None:
        kw["hydro"] = hydro
    return ns, gen.kh_config(abi, **kw)


def _specs(pkg):
    abi = pkg.abi
    return [
        _sod_member(pkg, 64, 5.0 / 3.0, 4.0, abi.PRECISION_FP64, 1),
        _sod_member(pkg, 40, 1.4, 2.0, abi.PRECISION_MIXED, 2),
        _kh_member(pkg, abi.PRECISION_FP64),
        _sod_member(pkg, 96, 1.3, 8.0, abi.PRECISION_MIXED, 3),
        _kh_member(pkg, abi.PRECISION_FP64, hydro=abi.HYDRO_CRKSPH),
        _sod_member(pkg, 32, 1.5, 3.0, abi.PRECISION_FP64, 4),
    ]


def test_batch_members_match_solo_runs(gpu_lib, pkg):
    specs = _specs(pkg)
    solo = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    mem = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    for s in solo:
        s.build_neighbors()
    batch = pkg.SPHBatch(mem)
    batch.build_neighbors()
    for s, m in zip(solo, mem):
        so, sn, sr = s.connectivity()
        mo, mn, mr = m.connectivity()
        assert np.array_equal(so, mo) and np.array_equal(sn, mn) and np.array_equal(sr, mr)
    assert batch.num_pairs() == sum(s.num_pairs() for s in solo)
    for s in solo:
        s.step(3)
    batch.step(3)
    for s, m in zip(solo, mem):
        assert s.time == m.time
        for k in STATE_KEYS:
            assert np.array_equal(s.field(k), m.field(k)), k
        for k in ("delta velocity hydro", "delta specific thermal energy", "new H"):
            assert np.array_equal(s.field(k), m.field(k)), k


def test_batch_evaluate_derivatives_matches_solo(gpu_lib, pkg):
    specs = _specs(pkg)[:4]
    solo = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    mem = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    for s in solo:
        s.build_neighbors()
        s.initialize()
        s.evaluateDerivatives()
    batch = pkg.SPHBatch(mem)
    batch.build_neighbors()
    batch.evaluateDerivatives()
    for s, m in zip(solo, mem):
        for k in ("delta velocity hydro", "delta specific thermal energy", "delta mass density",
                  "velocity gradient", "new H", "max viscous pressure"):
            assert np.array_equal(s.field(k), m.field(k)), k


def test_batch_launch_count_independent_of_members(gpu_lib, pkg):
    """One launch per stage: a step of 2 members and of 5 members of the same
    kind issue the same number of kernels (with the ghost passes as launches
    per pass; the automatic schedule runs them as one cooperative launch for
    batches of at most 4 members)."""
    abi = pkg.abi
    counts = []
    for nm in (2, 5):
        mem = []
        for k in range(nm):
            ns, cfg = _sod_member(pkg, 32 + 8 * k, 5.0 / 3.0, 4.0, abi.PRECISION_MIXED, 10 + k)
            mem.append(pkg.SPHHydro(cfg, ns))
        batch = pkg.SPHBatch(mem)
        batch.set_schedule("ghost passes", 1)
        batch.step(1)
        before = batch.kernel_launches()
        batch.step(1)
        counts.append(batch.kernel_launches() - before)
    assert counts[0] == counts[1]


def test_autotune_keeps_results(gpu_lib, pkg):
    """The autotuner picks schedules by timing; every schedule gives the same
    bits, so a tuned batch and an untuned solo run agree exactly.  Tuning
    leaves the derivatives evaluated at the current state, as
    evaluateDerivatives does."""
    specs = _specs(pkg)[:4]
    solo = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    mem = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    for s in solo:
        s.build_neighbors()
        s.initialize()
        s.evaluateDerivatives()
    batch = pkg.SPHBatch(mem)
    batch.build_neighbors()
    rep = batch.autotune()
    assert rep["neighbor walk"] in (1, 2) and rep["pair loop"] in (64, 128, 256)
    assert rep["neighbor cells"] in (1, 2) and rep["neighbor cells ms"][2] > 0
    assert all(v > 0 for v in rep["neighbor walk ms"].values())
    batch.step(2)
    for s in solo:
        s.step(2)
    for s, m in zip(solo, mem):
        for k in STATE_KEYS:
            assert np.array_equal(s.field(k), m.field(k)), k
    # per problem too: the tuned derivatives equal an untuned evaluation
    g = pkg.SPHHydro(specs[0][1], specs[0][0])
    r = pkg.SPHHydro(specs[0][1], specs[0][0])
    g.build_neighbors()
    rep = g.autotune()
    assert g.schedule("pair loop") == rep["pair loop"]
    r.build_neighbors()
    r.evaluateDerivatives()
    for k in ("delta velocity hydro", "delta specific thermal energy", "new H"):
        assert np.array_equal(g.field(k), r.field(k)), k


def test_graph_replayed_steps_match_eager(gpu_lib, pkg):
    """The whole RK2 step, rebuild included, as a captured CUDA graph (one
    capture, then replays with no host round trip) gives exactly the eager
    results, for a batch (SPH, mixed, CRKSPH members) and for a single
    problem."""
    specs = _specs(pkg)
    eager = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    mem = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    for e in eager:
        e.set_schedule("step graph", 0)
        e.step(4)
    batch = pkg.SPHBatch(mem)
    batch.set_schedule("step graph", 1)
    batch.step(4)
    for e, m in zip(eager, mem):
        assert e.time == m.time
        for k in STATE_KEYS:
            assert np.array_equal(e.field(k), m.field(k)), k
    ns, cfg = specs[1]
    a, g = pkg.SPHHydro(cfg, ns), pkg.SPHHydro(cfg, ns)
    a.set_schedule("step graph", 0)
    assert a.schedule("step graph") == 0
    a.step(3)
    g.step(3)
    assert g.schedule("step graph") == 1
    for k in STATE_KEYS:
        assert np.array_equal(a.field(k), g.field(k)), k
    assert g.pairs_evaluated() == a.pairs_evaluated()
    assert batch.pairs_evaluated() == sum(e.pairs_evaluated() for e in eager)
    # new state of the same layout: the next call replays the graph at once
    for h in (a, g):
        h.set_state(_State(h, 1.0))
        h.step(2)
    assert g.num_pairs() == a.num_pairs()
    for k in STATE_KEYS:
        assert np.array_equal(a.field(k), g.field(k)), k


class _State:
    """A node set read back from a problem, with H scaled."""

    def __init__(self, h, hscale):
        self.pos = h.field("position")
        self.vel = h.field("velocity")
        self.mass = h.field("mass")
        self.rho = h.field("mass density")
        self.eps = h.field("specific thermal energy")
        self.H = h.field("H") * hscale


@pytest.mark.parametrize("hydro", ["sph", "crksph"])
def test_graph_steps_regrow_after_overflow(gpu_lib, pkg, hydro):
    """Graph replays after new state that outgrows the buffers: the caller
    shrinks every H by 2/3 between calls (about 3.4x the neighbors), so the
    first replayed rebuild overflows its ghost, entry and list capacities; the
    gate skips the rest of that step, the library grows the buffers, takes
    the step eagerly (with the CRKSPH start-up volume new state needs) and
    captures again.  States, times and the pair counter equal eager steps bit
    for bit."""
    abi = pkg.abi
    ns, cfg = _kh_member(pkg, abi.PRECISION_FP64,
                         hydro=abi.HYDRO_CRKSPH if hydro == "crksph" else None)
    a, g = pkg.SPHHydro(cfg, ns), pkg.SPHHydro(cfg, ns)
    a.set_schedule("step graph", 0)
    pairs = 0
    for _ in range(4):
        a.step(1)
        pairs += a.num_pairs()
    g.step(4)
    assert g.pairs_evaluated() == a.pairs_evaluated() == pairs
    e0 = g.num_pairs()
    for h in (a, g):
        h.set_state(_State(h, 2.0 / 3.0))
    p0 = g.pairs_evaluated()
    per_step = []
    for _ in range(5):
        a.step(1)
        per_step.append(a.num_pairs())
    g.step(5)
    assert per_step[0] > 2 * e0          # the first rebuild after the new state outgrew the buffers
    assert g.time == a.time
    for k in STATE_KEYS:
        assert np.array_equal(a.field(k), g.field(k)), k
    assert g.pairs_evaluated() - p0 == sum(per_step)
    assert g.pairs_evaluated() == a.pairs_evaluated()
    so, sn, sr = a.connectivity()
    go, gn, gr = g.connectivity()
    assert np.array_equal(so, go) and np.array_equal(sn, gn) and np.array_equal(sr, gr)


def test_batch_of_mixed_sph_and_mixed_crk_members(gpu_lib, pkg):
    """Mixed-form SPH and CRKSPH members in one batch keep their own record
    layouts and kernels: each equals its solo run bit for bit."""
    abi = pkg.abi
    specs = [_sod_member(pkg, 48, 1.4, 3.0, abi.PRECISION_MIXED, 21),
             _kh_member(pkg, abi.PRECISION_MIXED, hydro=abi.HYDRO_CRKSPH),
             _kh_member(pkg, abi.PRECISION_MIXED),
             _sod_member(pkg, 40, 5.0 / 3.0, 2.0, abi.PRECISION_FP64, 22)]
    solo = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    mem = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    for s in solo:
        s.step(3)
    batch = pkg.SPHBatch(mem)
    batch.step(3)
    for s, m in zip(solo, mem):
        for k in STATE_KEYS:
            assert np.array_equal(s.field(k), m.field(k)), k


def test_batch_of_record_only_and_grad_h_members(gpu_lib, pkg):
    """In the RK2 step the members without grad-h keep their mid-point state
    in the records only (state0 holds the start velocity and the mid-point H
    and density), while grad-h members take the full state0 copy.  Both kinds
    in one batch, FP64 and mixed, compatible energy on and off: each member
    equals its solo run bit for bit."""
    abi = pkg.abi
    specs = [_sod_member(pkg, 48, 1.4, 3.0, abi.PRECISION_MIXED, 31),
             _sod_member(pkg, 40, 5.0 / 3.0, 2.0, abi.PRECISION_FP64, 32),
             _sod_member(pkg, 40, 1.5, 4.0, abi.PRECISION_FP64, 33),
             _sod_member(pkg, 48, 1.3, 2.5, abi.PRECISION_MIXED, 34),
             _kh_member(pkg, abi.PRECISION_MIXED)]
    specs[1][1].gradhCorrection = 1
    specs[3][1].gradhCorrection = 1
    specs[2][1].compatibleEnergyEvolution = 0
    specs[2][1].densityUpdate = abi.DENSITY_INTEGRATE
    solo = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    mem = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
    for s in solo:
        s.step(4)
    batch = pkg.SPHBatch(mem)
    batch.step(4)
    for s, m in zip(solo, mem):
        assert s.time == m.time
        for k in STATE_KEYS:
            assert np.array_equal(s.field(k), m.field(k)), k
        for k in ("delta velocity hydro", "delta specific thermal energy", "new H"):
            assert np.array_equal(s.field(k), m.field(k)), k


def test_batch_rejects_duplicates(gpu_lib, pkg):
    ns, cfg = _sod_member(pkg, 32, 5.0 / 3.0, 4.0, pkg.abi.PRECISION_FP64, 5)
    a = pkg.SPHHydro(cfg, ns)
    with pytest.raises(RuntimeError):
        pkg.SPHBatch([a, a])
