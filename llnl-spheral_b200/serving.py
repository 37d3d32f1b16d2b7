"""Serving: a continuous-batching request loop over the C-ABI server.

``Server`` wraps ``sphgpu_server_*`` (admission by device-memory footprint,
one batched RK2 step of every running simulation per tick, state resident on
the device).  ``poisson_trace`` draws a seeded request trace of
Kelvin-Helmholtz and Sod-type problems; ``serve`` replays a trace in real
time: requests are submitted when their arrival time has passed, the server
ticks while work remains, and each request's time to completion (arrival to
retirement) is recorded.
"""
import ctypes
import time

import numpy as np

from . import abi, generators

_P = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_P)


class Server:
    QUEUED, RUNNING, DONE, FAILED, CANCELLED = 0, 1, 2, 3, 4

    def __init__(self, budget_bytes, max_members=512):
        self.lib = abi.load_library()
        h = _P()
        abi.check(self.lib.sphgpu_server_create(float(budget_bytes), int(max_members), ctypes.byref(h)), self.lib)
        self.h = h
        self._n = {}

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.sphgpu_server_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, cfg, nodes, nsteps):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (nodes.pos, nodes.vel, nodes.mass, nodes.rho, nodes.eps, nodes.H)]
        rid = ctypes.c_int64()
        abi.check(self.lib.sphgpu_server_submit(self.h, ctypes.byref(cfg), nodes.n, *[_ptr(a) for a in arrs],
                                                int(nsteps), ctypes.byref(rid)), self.lib)
        self._n[rid.value] = nodes.n
        return rid.value

    def tick(self):
        r = ctypes.c_int32()
        q = ctypes.c_int32()
        abi.check(self.lib.sphgpu_server_tick(self.h, ctypes.byref(r), ctypes.byref(q)), self.lib)
        return r.value, q.value

    def cancel(self, rid):
        """Withdraw a queued or running request; it is reported finished as CANCELLED."""
        abi.check(self.lib.sphgpu_server_cancel(self.h, int(rid)), self.lib)

    def finished(self):
        ids = np.zeros(4096, dtype=np.int64)
        cnt = ctypes.c_int32()
        out = []
        while True:
            abi.check(self.lib.sphgpu_server_finished(self.h, _ptr(ids), ids.size, ctypes.byref(cnt)), self.lib)
            out.extend(ids[:cnt.value].tolist())
            if cnt.value < ids.size:
                return out

    def status(self, rid):
        st = ctypes.c_int32()
        steps = ctypes.c_int64()
        pairs = ctypes.c_int64()
        abi.check(self.lib.sphgpu_server_status(self.h, int(rid), ctypes.byref(st), ctypes.byref(steps),
                                                ctypes.byref(pairs)), self.lib)
        return st.value, steps.value, pairs.value

    def error(self):
        return self.lib.sphgpu_last_error().decode()

    def fetch(self, rid):
        n = self._n.pop(rid)
        out = {k: np.empty(n * c) for k, c in (("position", 3), ("velocity", 3), ("mass", 1),
                                                ("mass density", 1), ("specific thermal energy", 1), ("H", 6))}
        t = ctypes.c_double()
        abi.check(self.lib.sphgpu_server_fetch(self.h, int(rid), *[_ptr(out[k]) for k in
                                                                  ("position", "velocity", "mass", "mass density",
                                                                   "specific thermal energy", "H")],
                                               ctypes.byref(t)), self.lib)
        for k, c in (("position", 3), ("velocity", 3), ("H", 6)):
            out[k] = out[k].reshape(n, c)
        out["time"] = t.value
        return out

    def stats(self):
        out = np.zeros(8)
        abi.check(self.lib.sphgpu_server_stats(self.h, _ptr(out)), self.lib)
        keys = ("bytes_in_use", "peak_bytes", "budget", "pair_interactions", "ticks", "completed", "steps",
                "kernel_launches")
        return dict(zip(keys, out.tolist()))


def estimate_footprint(cfg, nodes):
    """Device bytes the server charges for a request before it runs (host only)."""
    lib = abi.load_library()
    pos = np.ascontiguousarray(nodes.pos, dtype=np.float64)
    H = np.ascontiguousarray(nodes.H, dtype=np.float64)
    out = ctypes.c_int64()
    abi.check(lib.sphgpu_estimate_footprint(ctypes.byref(cfg), nodes.n, _ptr(pos), _ptr(H), ctypes.byref(out)), lib)
    return out.value


def request_nodes(kind, n, seed, precision):
    """Node set and configuration of one request: a Kelvin-Helmholtz cube or
    a Sod-type tube (8:1:1 lattice) of about n nodes."""
    if kind == "kh":
        m = max(8, int(round(n ** (1.0 / 3.0))))
        ns = generators.kelvin_helmholtz(nx=m, ny=m, nz=m, seed=seed)
        cfg = generators.kh_config(abi, precision=precision)
    else:
        k = max(4, int(round((n / 8.0) ** (1.0 / 3.0))))
        box = ((0.0, 0.0, 0.0), (1.0, 1.0 / 8.0, 1.0 / 8.0))
        ns = generators.sod(nx=8 * k, ny=k, nz=k, box=box, seed=seed)
        cfg = generators.sod_config(abi, ns_box=box, precision=precision)
    return ns, cfg


def poisson_trace(rate=20.0, duration=60.0, nmin=8192, nmax=1048576, nsteps=200, seed=20261203, max_requests=None):
    """Seeded request trace: Poisson arrivals at `rate` per second over
    `duration` seconds, 50/50 KH and Sod, n log-uniform in [nmin, nmax]."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (max_requests is not None and len(out) >= max_requests):
            return out
        kind = "kh" if rng.random() < 0.5 else "sod"
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        out.append(dict(arrival=t, kind=kind, n=n, nsteps=nsteps, seed=int(rng.integers(1 << 30))))


def serve(trace, precision, budget_bytes=150e9, max_members=512, prepare=None, sleep=time.sleep, max_queued=64,
          prebuilt_nodes=48_000_000, lookahead=128):
    """Replay `trace` in real time on a fresh server.  Returns per-request
    times to completion (s), the makespan and the server statistics.

    Node sets are built before the replay starts (untimed) in arrival order
    while they hold at most `prebuilt_nodes` nodes (every request of a short
    trace); a background thread builds the rest in order, at most `lookahead`
    ahead of the submissions.  A request that has arrived and is built goes to
    the server while fewer than `max_queued` wait in the server's queue: the
    server admits its queue first come first served, head of line, so the
    admissions are those of an unbounded queue while host memory holds a
    bounded number of waiting node sets, however far a long trace outruns the
    device.  Times to completion run from each request's arrival."""
    import threading

    def make(k):
        r = trace[k]
        return prepare([r], precision)[0] if prepare else request_nodes(r["kind"], r["n"], r["seed"], precision)

    order = sorted(range(len(trace)), key=lambda k: trace[k]["arrival"])
    built = {}
    cv = threading.Condition()
    state = {"submitted": 0, "stop": False}
    nodes_built, nbuilt = 0, 0
    while nbuilt < len(order) and nodes_built < prebuilt_nodes:
        built[order[nbuilt]] = make(order[nbuilt])
        nodes_built += trace[order[nbuilt]]["n"]
        nbuilt += 1

    def producer(start):
        for idx in range(start, len(order)):
            with cv:
                while idx - state["submitted"] >= lookahead and not state["stop"]:
                    cv.wait(0.1)
                if state["stop"]:
                    return
            item = make(order[idx])
            with cv:
                built[order[idx]] = item
                cv.notify_all()

    worker = threading.Thread(target=producer, args=(nbuilt,), daemon=True)
    worker.start()
    srv = Server(budget_bytes, max_members)
    ids, ttc = {}, {}
    nxt, queued = 0, 0
    try:
        t0 = time.perf_counter()
        while len(ttc) < len(trace):
            now = time.perf_counter() - t0
            while nxt < len(order) and trace[order[nxt]]["arrival"] <= now and queued < max_queued:
                k = order[nxt]
                with cv:
                    item = built.pop(k, None)
                if item is None:
                    break                     # not built yet: keep the device busy meanwhile
                ns, cfg = item
                ids[srv.submit(cfg, ns, trace[k]["nsteps"])] = k
                nxt += 1
                queued += 1
                with cv:
                    state["submitted"] = nxt
                    cv.notify_all()
            running, queued = srv.tick()
            done_at = time.perf_counter() - t0
            for rid in srv.finished():
                k = ids[rid]
                st, _, _ = srv.status(rid)
                ttc[k] = done_at - trace[k]["arrival"] if st == Server.DONE else float("nan")
                if st == Server.DONE:
                    srv.fetch(rid)
            if running == 0 and queued == 0 and nxt < len(order):
                wait = trace[order[nxt]]["arrival"] - (time.perf_counter() - t0)
                if wait > 0:
                    sleep(wait)
                elif order[nxt] not in built:
                    sleep(0.001)              # the next request is still being built
        makespan = time.perf_counter() - t0
        stats = srv.stats()
    finally:
        with cv:
            state["stop"] = True
            cv.notify_all()
        worker.join()
        srv.close()
    return [ttc[k] for k in range(len(trace))], makespan, stats
