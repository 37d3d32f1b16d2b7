"""Placement of independent problems and requests on the GPUs of a node.

No GPU: the placement is host logic, computed identically on every rank.
The two-rank test runs world_size 2 over gloo on the CPU and checks that
the ranks' shares, computed independently, cover every item exactly once.
"""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _sharding():
    return importlib.import_module("llnl-spheral_b200.sharding")


def test_partition_covers_and_balances():
    sh = _sharding()
    rng = np.random.default_rng(3)
    costs = np.exp(rng.uniform(np.log(4096), np.log(262144), 256)).tolist()
    for world in (1, 2, 4, 8):
        r = sh.partition_by_cost(costs, world)
        assert sorted(k for q in range(world) for k in sh.local_items(r, q)) == list(range(len(costs)))
        loads = [sum(costs[k] for k in sh.local_items(r, q)) for q in range(world)]
        # LPT: no rank exceeds the mean by more than the largest item
        assert max(loads) <= sum(costs) / world + max(costs)
    assert sh.partition_by_cost(costs, 4) == sh.partition_by_cost(list(costs), 4)
    assert sh.partition_by_cost([], 3) == []
    with pytest.raises(ValueError):
        sh.partition_by_cost(costs, 0)


def test_routing_is_deterministic_and_spreads_bursts():
    sh = _sharding()
    arrivals = [0.0] * 8 + [10.0 + 0.1 * k for k in range(8)]
    costs = [1.0] * 16
    r = sh.route_requests(arrivals, costs, 4)
    assert r == sh.route_requests(list(arrivals), list(costs), 4)
    # a burst of 8 equal requests lands 2 per rank
    assert sorted(r[:8]) == [0, 0, 1, 1, 2, 2, 3, 3]
    # after the backlog has drained, spaced requests go to rank 0 first
    assert r[8] == 0
    assert sh.route_requests([], [], 2) == []


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, arrivals, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = _sharding()
        mine_b = sh.local_items(sh.partition_by_cost(costs, world), rank)
        mine_r = sh.local_items(sh.route_requests(arrivals, costs, world), rank)
        got = [None] * world
        dist.all_gather_object(got, (mine_b, mine_r))
        if rank == 0:
            q.put(got)
    finally:
        dist.destroy_process_group()


def test_two_ranks_compute_disjoint_covering_shares():
    rng = np.random.default_rng(11)
    costs = rng.uniform(1.0, 10.0, 40).tolist()
    arrivals = np.sort(rng.uniform(0.0, 5.0, 40)).tolist()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, arrivals, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for part in (0, 1):
        a, b = got[0][part], got[1][part]
        assert not set(a) & set(b)
        assert sorted(a + b) == list(range(40))
