"""Device memory reuse: the library's buffers come from a memory pool that
keeps freed blocks, so a new problem may land in memory another problem has
just used.  Results must not depend on what that memory held: the same
problem, created in fresh and in recycled memory, steps to the same bits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE_KEYS = ["position", "velocity", "mass density", "specific thermal energy", "H", "pressure", "sound speed"]


def _kh(pkg, precision, hydro=None, nz=8):
    gen, abi = pkg.generators, pkg.abi
    ns = gen.kelvin_helmholtz(nx=16, ny=16, nz=nz, box=((0, 0, 0), (1.0, 1.0, nz / 16.0)))
    kw = dict(xmax=(1.0, 1.0, nz / 16.0), precision=precision)
    if hydro is not None:
        kw["hydro"] = hydro
    return ns, gen.kh_config(abi, **kw)


def _run(pkg, ns, cfg, steps):
    h = pkg.SPHHydro(cfg, ns)
    h.step(steps)
    out = {k: h.field(k).copy() for k in STATE_KEYS}
    out["connectivity"] = [a.copy() for a in h.connectivity()]
    h.close()
    return out


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_recycled_memory_gives_identical_results(gpu_lib, pkg, precision):
    abi = pkg.abi
    prec = abi.PRECISION_MIXED if precision == "mixed" else abi.PRECISION_FP64
    ns, cfg = _kh(pkg, prec)
    first = _run(pkg, ns, cfg, 3)
    # other problems of other sizes, forms and precisions use and free memory
    for other_prec, hydro, nz in ((abi.PRECISION_FP64, None, 16), (abi.PRECISION_MIXED, abi.HYDRO_CRKSPH, 8),
                                  (abi.PRECISION_MIXED, None, 12)):
        o_ns, o_cfg = _kh(pkg, other_prec, hydro, nz)
        h = pkg.SPHHydro(o_cfg, o_ns)
        h.step(2)
        h.close()
    again = _run(pkg, ns, cfg, 3)
    for k in STATE_KEYS:
        assert np.array_equal(first[k], again[k]), k
    for a, b in zip(first["connectivity"], again["connectivity"]):
        assert np.array_equal(a, b)
