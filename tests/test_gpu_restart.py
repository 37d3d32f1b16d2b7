"""Checkpoint and restart (SPHHydroBase::dumpState / restoreState): a run
restarted from a checkpoint continues bit for bit, as the reference's
restart test requires (tests/Hydro/Sod/Sod-planar-1d.py:474-482)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

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
