"""Host-side serving logic on the CPU: the request trace and the admission
footprint estimate (no device call)."""
import numpy as np


def test_poisson_trace_is_seeded_and_shaped(pkg):
    s = pkg.serving
    a = s.poisson_trace(rate=20.0, duration=60.0, seed=7)
    b = s.poisson_trace(rate=20.0, duration=60.0, seed=7)
    assert a == b
    assert 900 < len(a) < 1500                        # ~ rate * duration
    arr = np.array([r["arrival"] for r in a])
    assert np.all(np.diff(arr) > 0) and arr[-1] <= 60.0
    n = np.array([r["n"] for r in a])
    assert n.min() >= 8192 and n.max() <= 1048576
    # log-uniform: the median is near the geometric mean of the bounds
    assert abs(np.log(np.median(n)) - 0.5 * (np.log(8192) + np.log(1048576))) < 0.3
    kinds = [r["kind"] for r in a]
    assert 0.4 < kinds.count("kh") / len(kinds) < 0.6


def test_footprint_estimate_scales_with_nodes(pkg):
    s = pkg.serving
    est = []
    for n in (4096, 32768, 262144):
        ns, cfg = s.request_nodes("sod", n, 1, 1)
        est.append(s.estimate_footprint(cfg, ns) / ns.n)
    # bytes per node: state, derivatives, records, cell list and ~120 B-spline neighbors
    assert all(1500 < e < 20000 for e in est), est
    # the ghost share falls as the tube grows
    assert est[0] > est[-1]
    ns, cfg = s.request_nodes("kh", 32768, 1, 1)
    kh = s.estimate_footprint(cfg, ns) / ns.n
    assert 800 < kh < est[1]                          # ~6 Wendland neighbors: fewer CSR bytes


def test_cancel_queued_requests_on_the_host(pkg):
    """Queue management needs no device: a queued request can be withdrawn,
    is reported finished as cancelled, and its fetch fails and releases it."""
    import pytest
    s = pkg.serving
    srv = s.Server(1e9, max_members=4)
    reqs = [s.request_nodes("sod", 4096, seed, 1) for seed in (1, 2, 3)]
    ids = [srv.submit(cfg, ns, 5) for ns, cfg in reqs]
    srv.cancel(ids[1])
    assert srv.status(ids[1])[0] == srv.CANCELLED
    assert srv.status(ids[0])[0] == srv.QUEUED and srv.status(ids[2])[0] == srv.QUEUED
    assert srv.finished() == [ids[1]]
    with pytest.raises(RuntimeError):
        srv.cancel(ids[1])                 # already finished
    with pytest.raises(RuntimeError):
        srv.fetch(ids[1])                  # cancelled: no result; the request is released
    with pytest.raises(RuntimeError):
        srv.status(ids[1])                 # unknown after release
    srv.cancel(ids[2])
    assert srv.finished() == [ids[2]]
    srv.close()
