"""Checkpoint and restart (SPHHydroBase::dumpState / restoreState): a run
restarted from its restart file continues bit for bit, as the reference's
restart test requires (tests/Hydro/Sod/Sod-planar-1d.py:474-482); the file
is the reference's own layout (RestartRegistrar::dumpState through
FlatFileIO), checked against restart files the reference wrote
(tests/golden/reference_restart_*) and, where the reference's checker was
built here (oracle/_ref/ref_sph), read back by the reference itself."""
import glob
import os
import subprocess

import numpy as np
import pytest

import flatfile
from conftest import ROOT, normwise

pytestmark = pytest.mark.gpu

FIXTURES = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "reference_restart_*.npz")))
IDS = [os.path.basename(p)[len("reference_restart_"):-4] for p in FIXTURES]
REF_SPH = os.path.join(ROOT, "oracle", "_ref", "ref_sph")

STATE_KEYS = ["position", "velocity", "mass density", "specific thermal energy", "H", "pressure", "sound speed"]


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


@pytest.mark.parametrize("which", ["sod", "sod_mixed", "kh", "kh_crk"])
def test_restart_continues_bit_for_bit(gpu_lib, pkg, which, tmp_path):
    ns, cfg = _case(pkg, which)
    straight = pkg.SPHHydro(cfg, ns)
    straight.step(6)
    first = pkg.SPHHydro(cfg, ns)
    first.step(3)
    t3 = first.time
    path = tmp_path / "restart.bin"
    first.dumpState(str(path))
    first.close()
    resumed = pkg.SPHHydro(cfg, n=ns.n)
    resumed.restoreState(str(path))
    assert resumed.time == t3                 # the time comes back with the image
    resumed.step(3)
    assert resumed.time == straight.time
    for k in STATE_KEYS:
        assert np.array_equal(resumed.field(k), straight.field(k)), k
    for k in ("delta velocity hydro", "delta specific thermal energy"):
        assert np.array_equal(resumed.field(k), straight.field(k)), k


def test_restore_rejects_mismatched_images(gpu_lib, pkg):
    ns, cfg = _case(pkg, "sod")
    a = pkg.SPHHydro(cfg, ns)
    a.step(1)
    image = a.checkpoint()
    other_ns, other_cfg = _case(pkg, "kh_crk")        # same node count, CRKSPH layout
    b = pkg.SPHHydro(other_cfg, other_ns)
    with pytest.raises(RuntimeError, match="does not match"):
        b.restore(image)
    with pytest.raises(RuntimeError, match="truncated"):
        a.restore(image[:len(image) // 2])
    with pytest.raises(RuntimeError, match="not a checkpoint"):
        a.restore(b"\0" * len(image))
    a.restore(image)                     # the problem stays usable
    a.step(1)


def _fixture(pkg, path):
    d = np.load(path)
    cfg = pkg.abi.SphConfig.from_buffer_copy(d["input/config"].tobytes())
    nodes = pkg.generators.NodeSet(d["input/position"], d["input/velocity"], d["input/mass"],
                                   d["input/mass density"], d["input/specific thermal energy"], d["input/H"], None)
    return d, cfg, nodes


def _run_to_dump(pkg, cfg, nodes, nsteps):
    """The reference checker's sequence: connectivity, one evaluation at the
    start time, then the RK2 steps."""
    h = pkg.SPHHydro(cfg, nodes)
    h.build_neighbors()
    h.initialize()
    h.evaluateDerivatives()
    h.step(nsteps)
    return h


def _same_values(ours, ref, skip=("/work",)):
    """Entries path by path in the same order; values bit-equal, or within
    1e-12 of the field's largest magnitude (the cube root of the ideal-H
    moment, CUDA pow against glibc pow, reaches the state after a step)."""
    assert [p for p, _ in ours] == [p for p, _ in ref]
    for (p, a), (_, b) in zip(ours, ref):
        if p.endswith(skip):
            continue
        if p.endswith("/NodeListNames") or p.endswith("/name"):
            assert a == b, p
            continue
        va, vb = flatfile.numbers(a), flatfile.numbers(b)
        assert va.size == vb.size, p
        if not np.array_equal(va, vb):
            assert normwise(va, vb) <= 1e-12, p


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_dump_matches_the_reference_file(gpu_lib, pkg, path, tmp_path):
    """Same objects, keys, order and values as the reference's restart file
    after the same steps of the same node set."""
    d, cfg, nodes = _fixture(pkg, path)
    h = _run_to_dump(pkg, cfg, nodes, int(d["input/nsteps"]))
    h.dumpState(tmp_path / "ours.txt")
    ours = flatfile.entries((tmp_path / "ours.txt").read_bytes())
    _same_values(ours, flatfile.entries(d["restart"].tobytes()))


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_restore_the_reference_file(gpu_lib, pkg, path, tmp_path):
    """A problem restored from the reference's own restart file continues as
    the reference continued from it (RestartRegistrar::restoreState, then
    the same RK2 steps): within 1e-12."""
    d, cfg, nodes = _fixture(pkg, path)
    f = tmp_path / "ref.txt"
    f.write_bytes(d["restart"].tobytes())
    h = pkg.SPHHydro(cfg, n=nodes.n)
    h.restoreState(f)
    t, last = h.step(int(d["input/nmore"]))
    tr, dtr = d["cont/time_dt"][-2:]
    assert abs(t - tr) <= 1e-12 * tr and abs(last - dtr) <= 1e-12 * dtr
    for key in STATE_KEYS:
        assert normwise(h.field(key).ravel(), d["cont/" + key]) <= 1e-12, key


@pytest.mark.skipif(not os.path.exists(REF_SPH), reason="reference checker not built here (oracle/build_ref.py)")
@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_reference_reads_our_file(gpu_lib, pkg, path, tmp_path):
    """The reference restores a file this library wrote (its FlatFileIO and
    RestartRegistrar::restoreState) and continues within 1e-12 of the run
    this library continues from the same file."""
    d, cfg, nodes = _fixture(pkg, path)
    nsteps, nmore = int(d["input/nsteps"]), int(d["input/nmore"])
    h = _run_to_dump(pkg, cfg, nodes, nsteps)
    f = tmp_path / "ours.txt"
    h.dumpState(f)
    h.step(nmore)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as out:
        out.write(np.int64(nodes.n).tobytes())
        out.write(np.int64(nmore).tobytes())
        out.write(bytes(cfg))
        for a in (nodes.pos, nodes.vel, nodes.mass, nodes.rho, nodes.eps, nodes.H):
            out.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
    (tmp_path / "cont" / "steps").mkdir(parents=True)
    subprocess.check_call([REF_SPH, "--restart-load", str(inp), str(f), str(tmp_path / "cont")],
                          stdout=subprocess.DEVNULL)
    for key in STATE_KEYS:
        ref = np.fromfile(tmp_path / "cont" / "steps" / (key + ".f64"), dtype="<f8")
        assert normwise(h.field(key).ravel(), ref) <= 1e-12, key
