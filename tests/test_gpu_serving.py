"""Serving: continuous batching with footprint admission.

Requests arrive while others run; each result must be exactly what the
request gives alone (the batched step does the member's own arithmetic in
its own order), the device-memory footprint must never exceed the budget,
and a request larger than the budget must fail cleanly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = [("position", "position"), ("velocity", "velocity"), ("mass density", "mass density"),
        ("specific thermal energy", "specific thermal energy"), ("H", "H")]


def _requests(pkg, precision):
    serving = pkg.serving
    specs = [("kh", 4096, 3, 11), ("sod", 2048, 5, 12), ("sod", 8192, 2, 13), ("kh", 1000, 4, 14),
             ("sod", 4000, 3, 15), ("kh", 2744, 2, 16)]
    out = []
    for kind, n, nsteps, seed in specs:
        ns, cfg = serving.request_nodes(kind, n, seed, precision)
        out.append((ns, cfg, nsteps))
    return out


def _solo(pkg, ns, cfg, nsteps):
    g = pkg.SPHHydro(cfg, ns)
    g.step(nsteps)
    return {k: g.field(k) for k, _ in KEYS}, g.time


def _run_server(pkg, reqs, budget, arrivals):
    """Submit request k before tick arrivals[k] (ticks count from 0)."""
    srv = pkg.serving.Server(budget, max_members=64)
    ids, results, tick = {}, {}, 0
    pending = sorted(range(len(reqs)), key=lambda k: arrivals[k])
    peak = 0.0
    while len(results) < len(reqs):
        while pending and arrivals[pending[0]] <= tick:
            k = pending.pop(0)
            ns, cfg, nsteps = reqs[k]
            ids[srv.submit(cfg, ns, nsteps)] = k
        srv.tick()
        tick += 1
        peak = max(peak, srv.stats()["bytes_in_use"])
        for rid in srv.finished():
            st, steps, pairs = srv.status(rid)
            results[ids[rid]] = (st, srv.fetch(rid) if st == srv.DONE else None, steps)
        assert tick < 200
    stats = srv.stats()
    srv.close()
    return results, stats, peak


@pytest.mark.parametrize("precision", [0, 1])
def test_served_results_equal_solo_runs(gpu_lib, pkg, precision):
    reqs = _requests(pkg, precision)
    arrivals = [0, 0, 1, 2, 2, 4]          # later requests join while earlier ones run
    results, stats, peak = _run_server(pkg, reqs, 40e9, arrivals)
    assert stats["completed"] == len(reqs)
    for k, (ns, cfg, nsteps) in enumerate(reqs):
        st, out, steps = results[k]
        assert st == 2 and steps == nsteps
        ref, t = _solo(pkg, ns, cfg, nsteps)
        assert out["time"] == t
        for key, _ in KEYS:
            assert np.array_equal(out[key], ref[key]), (k, key)


def test_admission_respects_budget(gpu_lib, pkg):
    reqs = _requests(pkg, 1)
    arrivals = [0] * len(reqs)
    # a budget that holds about two of these requests at a time
    est = [pkg.serving.estimate_footprint(cfg, ns) for ns, cfg, _ in reqs]
    budget = 2.2 * max(est)
    results, stats, peak = _run_server(pkg, reqs, budget, arrivals)
    assert stats["completed"] == len(reqs)
    assert stats["peak_bytes"] <= budget
    assert peak <= budget
    assert all(results[k][0] == 2 for k in range(len(reqs)))


def test_oversized_request_fails_cleanly(gpu_lib, pkg):
    reqs = _requests(pkg, 1)[:2]
    results, stats, _ = _run_server(pkg, reqs, 1.0e6, [0, 0])
    assert all(results[k][0] == 3 for k in range(2))
    assert stats["completed"] == 0


def test_cancel_a_running_request(gpu_lib, pkg):
    """A request cancelled while it runs gives its memory back at once; the
    requests running beside it finish with the results they give alone."""
    reqs = _requests(pkg, 1)[:3]
    srv = pkg.serving.Server(40e9, max_members=64)
    ids = [srv.submit(cfg, ns, nsteps) for ns, cfg, nsteps in reqs]
    srv.tick()
    before = srv.stats()["bytes_in_use"]
    assert srv.status(ids[1])[0] == srv.RUNNING
    srv.cancel(ids[1])
    assert srv.stats()["bytes_in_use"] < before
    done = {}
    for _ in range(20):
        srv.tick()
        for rid in srv.finished():
            done[rid] = srv.status(rid)[0]
        if len(done) == 3:
            break
    assert done[ids[1]] == srv.CANCELLED
    with pytest.raises(RuntimeError):
        srv.fetch(ids[1])
    for k in (0, 2):
        assert done[ids[k]] == srv.DONE
        out = srv.fetch(ids[k])
        ns, cfg, nsteps = reqs[k]
        ref, t = _solo(pkg, ns, cfg, nsteps)
        for key, _ in KEYS:
            assert np.array_equal(out[key], ref[key]), (k, key)
    srv.close()
