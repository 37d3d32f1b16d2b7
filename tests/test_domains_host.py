"""Slab domain decomposition, host side (no GPU): the periodic slab geometry
and, over world_size 2 gloo ranks on the CPU, the halo each rank receives
(DistributedSlabs.exchange_rows: extents by all_gather, rows by send/recv)
against the halo computed from the whole node set."""
import datetime
import importlib
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _mods():
    pkg = importlib.import_module("llnl-spheral_b200")
    return pkg, importlib.import_module("llnl-spheral_b200.domains")


def test_periodic_slab_geometry():
    _, dm = _mods()
    x = np.array([0.05, 0.45, 0.55, 0.95, 0.999])
    assert list(dm.slab_of(x, 2, 0.0, 1.0)) == [0, 0, 1, 1, 1]
    g = dm.periodic_gap(x, 0.0, 0.5, 1.0)
    assert np.allclose(g, [0.0, 0.0, 0.05, 0.05, 0.001])
    # an interval reaching below the box start wraps
    assert np.allclose(dm.periodic_gap(np.array([0.98, 0.995, 0.7]), -0.01, 0.5, 1.0), [0.01, 0.0, 0.2])
    H = np.tile([10.0, 0.0, 0.0, 20.0, 0.0, 40.0], (3, 1))
    assert np.isclose(dm.max_h(H), 0.1)


def _problem(pkg):
    gen, abi = pkg.generators, pkg.abi
    ns = gen.kelvin_helmholtz(nx=16, ny=8, nz=4, box=((0, 0, 0), (1.0, 0.5, 0.25)))
    cfg = gen.kh_config(abi, xmax=(1.0, 0.5, 0.25))
    return ns, cfg


def expected_halo(dm, ns, cfg, world, rank):
    owner = dm.slab_of(ns.pos[:, 0], world, cfg.xmin[0], cfg.xmax[0])
    L = cfg.xmax[0] - cfg.xmin[0]
    reach = dm.KERNEL_EXTENT * dm.max_h(ns.H)
    lo, hi = rank * L / world, (rank + 1) * L / world
    mine = np.nonzero(owner == rank)[0]
    widen = dm.periodic_gap(ns.pos[mine, 0], lo, hi, L).max()
    gap = dm.periodic_gap(ns.pos[:, 0], lo - widen, hi + widen, L)
    return np.nonzero((owner != rank) & (gap <= dm.halo_depth(cfg) * reach))[0]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pkg, dm = _mods()
        ns, cfg = _problem(pkg)
        ds = dm.DistributedSlabs(cfg, ns)
        rows = ds.exchange_rows()
        got = np.sort(np.concatenate([r[:, 0] for r in rows]).astype(np.int64))
        # the rows carry the senders' state of those nodes
        allrows = np.concatenate(rows)
        order = np.argsort(allrows[:, 0])
        ok_state = np.array_equal(allrows[order, 1:4], ns.pos[got])
        q.put((rank, got.tolist(), bool(ok_state), ds.domain.gid.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_receive_the_halo():
    pkg, dm = _mods()
    ns, cfg = _problem(pkg)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = []
    for rank, got, ok_state, gid in sorted(res):
        assert got == expected_halo(dm, ns, cfg, 2, rank).tolist()
        assert ok_state
        owned += gid
    assert sorted(owned) == list(range(ns.n))       # every node owned once
