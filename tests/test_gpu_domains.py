"""Slab domain decomposition on one GPU: `world` slab domains of one problem
emulated in one process (SlabDecomposition: the same phases and data as one
rank per GPU, the exchange a transpose of the send lists).  Against the
single-domain run of the same node set:
  - every node's neighbor set, as (global node, periodic image), is the
    single-domain one (the slab boundaries included);
  - the derivatives at the start time and the state after RK2 steps agree
    within 1e-12 normwise (only the order of the pair sums differs);
  - the time steps agree."""
import importlib

import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu

STATE = ["position", "velocity", "mass density", "specific thermal energy", "H"]
DERIVS = ["delta velocity hydro", "delta specific thermal energy", "delta mass density", "new H",
          "velocity gradient"]


def _case(pkg, name):
    gen, abi = pkg.generators, pkg.abi
    if name == "sod_gradh":
        box = ((0.0, 0.0, 0.0), (1.0, 0.25, 0.25))
        ns = gen.sod(nx=32, ny=8, nz=8, box=box, jitter=0.05)
        ns.vel[:, 0] = 0.05 * np.sin(2 * np.pi * ns.pos[:, 0])
        return ns, gen.sod_config(abi, ns_box=box, gradhCorrection=1)
    ns = gen.kelvin_helmholtz(nx=16, ny=16, nz=8, box=((0, 0, 0), (1.0, 1.0, 0.5)))
    kw = {"hydro": abi.HYDRO_CRKSPH} if name == "crk_kh" else {}
    return ns, gen.kh_config(abi, xmax=(1.0, 1.0, 0.5), **kw)


def _rows(h, gid, cfg, count):
    off, nb, root = h.connectivity()
    gpos = h.ghost_positions()
    pos = h.field("position")
    L = np.array(cfg.xmax) - np.array(cfg.xmin)
    out = []
    for i in range(count):
        row = []
        for j in nb[off[i]:off[i + 1]]:
            if j < h.n:
                row.append((int(gid[j]), 0, 0, 0))
            else:
                r = int(root[j - h.n])
                s = np.rint((gpos[j - h.n] - pos[r]) / L).astype(int)
                row.append((int(gid[r]), int(s[0]), int(s[1]), int(s[2])))
        out.append(sorted(row))
    return out


@pytest.mark.parametrize("name,world", [("kh", 2), ("kh", 3), ("sod_gradh", 2), ("crk_kh", 2)])
def test_slab_domains_match_single_domain(gpu_lib, pkg, name, world):
    dm = importlib.import_module("llnl-spheral_b200.domains")
    ns, cfg = _case(pkg, name)
    one = pkg.SPHHydro(cfg, ns)
    one.build_neighbors()
    one.initialize()
    one.evaluateDerivatives()
    dd = dm.SlabDecomposition(cfg, ns, world)
    dd.initialize()
    # neighbor sets across the slab boundaries
    single = _rows(one, np.arange(ns.n), cfg, ns.n)
    got = [None] * ns.n
    for d in dd.domains:
        assert d.halo_gid.size > 0
        for gid, row in zip(d.gid, d.rows_global()):
            got[gid] = row
    assert got == single
    for key in DERIVS:
        assert normwise(dd.field(key, ns.n).ravel(), one.field(key).ravel()) <= 1e-12, key
    t, last = one.step(3)
    dd.step(3)
    for d in dd.domains:
        assert abs(d.time - t) <= 1e-12 * t and abs(d.last_dt - last) <= 1e-12 * last
    for key in STATE:
        assert normwise(dd.field(key, ns.n).ravel(), one.field(key).ravel()) <= 1e-12, key
    dd.close()
