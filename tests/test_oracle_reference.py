"""The oracle against the reference's own SPH / CRKSPH path, executed.

tests/golden/reference_sph_<case>.npz hold what the reference's
SPHHydroBase / CRKSPHHydroBase, ConnectivityMap, PeriodicBoundary and
CheapSynchronousRK2 (compiled from the reference's sources by
oracle/build_ref.py and driven by oracle/refshim/ref_sph.cc, see
tests/golden/make_golden.py) computed on small seeded node sets.  The oracle
must reproduce every number bit for bit: the ghosts and the ConnectivityMap,
every derivative field of one evaluateDerivatives, the pair accelerations,
the hydro time-step vote, and the state after the RK2 steps.

The reference culls unused ghosts (Integrator::setGhostNodes,
src/Integrator/Integrator.cc:494-594) and the oracle does not, so ghost
indices differ; neighbors are compared as (root node, ghost position) in row
order, which culling preserves.
"""
import glob
import hashlib
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "reference_sph_*.npz")))
CASES = [os.path.basename(f)[len("reference_sph_"):-4] for f in FIXTURES]


class Fixture:
    def __init__(self, pkg, name):
        self.d = np.load(os.path.join(HERE, "golden", "reference_sph_%s.npz" % name))
        d = self.d
        self.cfg = pkg.abi.SphConfig.from_buffer_copy(d["input/config"].tobytes())
        self.nsteps = int(d["input/nsteps"])
        self.nodes = pkg.generators.NodeSet(d["input/position"], d["input/velocity"], d["input/mass"],
                                            d["input/mass density"], d["input/specific thermal energy"],
                                            d["input/H"], None)
        self.n = self.nodes.n

    def __getitem__(self, k):
        return self.d[k]

    def eval_keys(self):
        return [k[5:] for k in self.d.files if k.startswith("eval/") and k not in
                ("eval/hydro dt", "eval/pair accelerations sha256", "eval/pair accelerations size")]

    def rows(self):
        """Per internal node: its neighbors as (root, x, y, z), x = y = z = 0 for internal ones."""
        return canonical_rows(self.n, self.d["conn_offsets"], self.d["conn_neighbors"], self.d["ghost_root"],
                              self.d["ghost_position"].reshape(-1, 3))


def canonical_rows(n, offsets, neighbors, ghost_root, ghost_position):
    out = []
    for i in range(n):
        row = []
        for j in neighbors[offsets[i]:offsets[i + 1]]:
            if j < n:
                row.append((int(j), 0.0, 0.0, 0.0))
            else:
                g = j - n
                row.append((int(ghost_root[g]),) + tuple(float(c) for c in ghost_position[g]))
        out.append(row)
    return out


def pair_acc_digest(a):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).digest(), dtype=np.uint8)


@pytest.fixture(scope="module", params=CASES)
def case(request, pkg):
    return request.param, Fixture(pkg, request.param)


def test_fixtures_present():
    assert len(CASES) >= 10


def test_oracle_matches_reference(case, oracle_mod):
    name, fx = case
    o = oracle_mod.OracleProblem(fx.cfg, fx.nodes)
    o.build_neighbors()
    o.initialize()
    off, nb, root = o.connectivity()
    assert canonical_rows(fx.n, off, nb, root, o.ghost_positions()) == fx.rows()
    o.evaluate_derivatives()
    for key in fx.eval_keys():
        assert np.array_equal(o.field(key).ravel(), fx["eval/" + key]), key
    if fx.cfg.compatibleEnergyEvolution:
        pa = np.zeros(int(fx["eval/pair accelerations size"]))
        import ctypes
        o.L.orc_get_pair_accelerations(o.h, pa.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(pair_acc_digest(pa), fx["eval/pair accelerations sha256"])
    assert o.dt() == fx["eval/hydro dt"][0]
    t, dt = o.step(fx.nsteps)
    assert (t, dt) == tuple(fx["steps/time_dt"][-2:])
    for key in ("position", "velocity", "mass density", "specific thermal energy", "H", "pressure", "sound speed"):
        assert np.array_equal(o.field(key).ravel(), fx["steps/" + key]), key
    if fx.cfg.hydro == 1:
        assert np.array_equal(o.field("node volume").ravel(), fx["steps/node volume"])


def test_fixtures_match_a_fresh_reference_run(pkg):
    """Where the reference tree is present (the development container), the
    committed fixtures are what the reference computes today."""
    import importlib
    import sys
    build_ref = importlib.import_module("build_ref")
    if not os.path.isdir(build_ref.reference_src()):
        pytest.skip("reference tree not present")
    sys.path.insert(0, os.path.join(HERE, "golden"))
    mg = importlib.import_module("make_golden")
    ref_sph, _ = build_ref.build()
    cs = mg.cases(pkg)
    for name in ("sod", "crk_kh"):
        ns, cfg, nsteps = cs[name]
        r = mg.run_reference(ref_sph, cfg, ns, nsteps)
        fx = Fixture(pkg, name)
        assert bytes(fx.cfg) == bytes(cfg)
        for k, v in r.items():
            if k == "eval/pair accelerations":
                assert np.array_equal(pair_acc_digest(v), fx["eval/pair accelerations sha256"])
            else:
                assert np.array_equal(v, fx[k]), k


IDEALH = sorted(glob.glob(os.path.join(HERE, "golden", "reference_idealh_*.npz")))


def idealh_fixture(pkg, path):
    d = np.load(path)
    cfg = pkg.abi.SphConfig.from_buffer_copy(d["input/config"].tobytes())
    nodes = pkg.generators.NodeSet(d["input/position"], d["input/velocity"], d["input/mass"], d["input/mass density"],
                                   d["input/specific thermal energy"], d["input/H"], None)
    return d, cfg, nodes


@pytest.mark.parametrize("path", IDEALH, ids=[os.path.basename(p)[:-4] for p in IDEALH])
def test_oracle_iterate_ideal_h_matches_reference(pkg, oracle_mod, path):
    """The reference's iterateIdealH (src/Utilities/iterateIdealH.cc, run by
    oracle/_ref/ref_sph as SpheralController.iterateIdealH calls it): the
    oracle's relaxed H is bit-equal, its iteration count equal, and its last
    change equal to the six digits the reference prints."""
    d, cfg, nodes = idealh_fixture(pkg, path)
    o = oracle_mod.OracleProblem(cfg, nodes)
    itr, dh = o.iterate_ideal_h(int(d["input/max_iterations"]), float(d["input/tolerance"]))
    assert itr == int(d["iterations"]) and 1 < itr < int(d["input/max_iterations"])
    assert abs(dh - float(d["max_delta_h_printed"])) <= 1e-5 * dh
    assert np.array_equal(o.field("H").ravel(), d["H"])
