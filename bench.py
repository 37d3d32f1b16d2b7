#!/usr/bin/env python
"""Benchmark of the B200 SPH hydro path on the Kelvin-Helmholtz configuration.

Workload (the configuration the headline metric is quoted on): 3-D
Kelvin-Helmholtz in the periodic unit cube, 128^3 = 2,097,152 nodes, +-0.01 dx
seeded jitter, Wendland C4 TableKernel(1000), nPerh 1.35, Monaghan-Gingold
Cl = Cq = 1, compatible energy, RigorousSumDensity, IdealH, Courant dt
(cfl 0.25).  Seeded synthetic node sets stand in for the reference's driver.

A step is one CheapSynchronousRK2 step on the device: periodic ghosts and
ConnectivityMap rebuilt, dt selected, mid-point derivatives, compatible-energy
and state updates, sum density, boundary wrap.  The metric is
pair-interactions/s (unordered neighbor pairs per derivative evaluation,
the reference's ncalc, times steps, over time).  The headline `value` is the
plain FP64 form, the reference's own arithmetic; the mixed FP32-pair form,
its ratio to FP64 and p50/p99 step latency of both are in the same line.

--impl reference times the reference's own CPU path (SPHHydroBase +
CheapSynchronousRK2 compiled from its sources into oracle/_ref/ref_sph; the
oracle restatement where that binary is absent) on all host cores, one
process per core on a z-slab of the same lattice.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import importlib
import json
import multiprocessing as mp
import os
import platform
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "pair-interactions/s"
WORKLOAD = ("Kelvin-Helmholtz 3-D periodic unit cube, 128^3 = 2,097,152 nodes, Wendland C4 "
            "TableKernel(1000), nPerh 1.35, MonaghanGingold Cl=Cq=1, compatible energy, "
            "RigorousSumDensity, IdealH, Courant dt (cfl 0.25); H relaxed to the ideal smoothing scale at "
            "start-up (iterateIdealH, untimed); one CheapSynchronousRK2 step per step")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=128, help="lattice size per axis (default: the full workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=200,
                    help="RK2 steps of the mixed-vs-FP64 error and energy-drift line (0: skip)")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the Sod (plain FP64) and CRKSPH Kelvin-Helmholtz lines")
    ap.add_argument("--kernel-survey", action="store_true",
                    help="no timing: run every kernel of the SPH and CRKSPH steps once on small problems "
                         "(the workload of the per-kernel profile) and exit")
    ap.add_argument("--batch", type=int, default=256, help="problems in the batched-ensemble line (0: skip)")
    ap.add_argument("--serving", type=float, default=2.0,
                    help="seconds of Poisson arrivals in the serving line (0: skip; 60 = the full trace)")
    ap.add_argument("--serving-steps", type=int, default=20, help="RK2 steps per served request (full: 200)")
    return ap.parse_args()


# Algorithmic bytes of one plain-FP64 evaluateDerivatives (record pack + pair
# kernel): the pack reads 136 B of state per internal node (position,
# velocity, m, rho, cs, P, omega, H) and writes a 160-byte pair record per
# node and ghost; the pair kernel reads those records, writes 54 derivative
# doubles per internal node (432 B; the reference's "internal velocity
# gradient" and "local M" equal the velocity gradient and M for one NodeList
# and are not stored twice), reads 4 B of CSR index and writes 24 B of FP64
# pair acceleration per directed entry.
def eval_alg_bytes_fp64(nodes, ghosts, entries):
    return nodes * 136 + 2 * (nodes + ghosts) * 160 + nodes * 432 + 28 * entries


# The same for the mixed form: 112-byte records, FP32 pair accelerations.
def eval_alg_bytes_mixed(nodes, ghosts, entries):
    return nodes * 136 + 2 * (nodes + ghosts) * 112 + nodes * 432 + 16 * entries


# DRAM traffic (read + write) measured by ncu on Kelvin-Helmholtz 96^3
# (884,736 nodes, 56,456 ghosts, 5,363,712 entries) for the record pack and
# the pair kernel of each form; scaled to other sizes by the algorithmic
# bytes (all three units grow together).
EVAL_TRAFFIC_96 = {"fp64": 155681536 + 107269376 + 180020480 + 449962752,
                   "mixed": 150498816 + 67565056 + 190594816 + 386470912}
EVAL_UNITS_96 = (884736, 56456, 5363712)


def kh_problem(pkg, nx, nz=None, seed=20261203):
    gen, abi = pkg.generators, pkg.abi
    nz = nz or nx
    ns = gen.kelvin_helmholtz(nx=nx, ny=nx, nz=nz, box=((0, 0, 0), (1.0, 1.0, nz / nx)), seed=seed)
    cfg = gen.kh_config(abi, xmax=(1.0, 1.0, nz / nx))
    return ns, cfg


# The controller's start-up relaxes H to the ideal smoothing scale before the
# run (SpheralController's iterateInitialH, on by default): maximum
# iterations and tolerance of that iterateIdealH.
IDEAL_H = (50, 1.0e-4)


def relax_h(pkg, ns, cfg):
    """ns.H relaxed to the ideal smoothing scale on the device
    (sphgpu_iterate_ideal_h), as the reference's start-up does; untimed set-up."""
    h = pkg.SPHHydro(cfg, ns)
    h.iterateIdealH(*IDEAL_H)
    ns.H = np.ascontiguousarray(h.field("H"))
    h.close()
    return ns


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            # line-buffered output (stdbuf) so that no sample is lost when the
            # sampler is stopped
            pre = ["stdbuf", "-oL"] if shutil.which("stdbuf") else []
            self.proc = subprocess.Popen(pre + ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                                "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # the sampler takes a moment to start: wait (at most 5 s) for its
        # first sample, so that it covers the whole timed region
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.12)          # a sample after the end of the timed region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for nm, v in zip(names, r[4:8]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(nm)
            except Exception:
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def allmax(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def measure_steps(pkg, ns, cfg, precision, steps, warmup, world, clocks=None, graph=True):
    """K RK2 steps, one sphgpu_step_rk2 call per step, with CUDA events
    around each step (per-step latency); `graph`: each call one replay of the
    captured whole-step graph (the default schedule), else eager launches."""
    import torch
    c = cfg.copy()
    c.precision = precision
    h = pkg.SPHHydro(c, ns)
    h.set_schedule("step graph", 1 if graph else 0)
    h.build_neighbors()
    h.evaluateDerivatives()          # derivatives at t = 0 feed the first predictor
    stream = torch.cuda.ExternalStream(h.stream())
    for _ in range(warmup):
        h.step(1)
    h.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    pairs = 0
    l0 = h.kernel_launches()
    if clocks:
        clocks.start()
    ev[0].record(stream)
    for k in range(steps):
        h.step(1)
        pairs += h.num_pairs()
        ev[k + 1].record(stream)
    h.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    barrier(world)
    launches = h.kernel_launches() - l0
    per = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
    total_ms = ev[0].elapsed_time(ev[steps])
    return h, {"total_ms": total_ms, "per_step_ms": per, "pairs": pairs, "launches": launches, "clocks": clk}


def measure_steps_graph(pkg, ns, cfg, precision, steps, warmup, world, clocks=None):
    """K RK2 steps in ONE sphgpu_step_rk2 call with the "step graph" schedule:
    the whole step (rebuild included) is a captured CUDA graph replayed K
    times with no host round trip; pairs from the device-side pair counter."""
    import torch
    c = cfg.copy()
    c.precision = precision
    h = pkg.SPHHydro(c, ns)
    h.set_schedule("step graph", 1)
    h.build_neighbors()
    h.evaluateDerivatives()
    stream = torch.cuda.ExternalStream(h.stream())
    for _ in range(max(warmup, 3)):      # eager step, capture + replay, replay
        h.step(1)
    h.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    p0 = h.pairs_evaluated()
    l0 = h.kernel_launches()
    if clocks:
        clocks.start()
    a.record(stream)
    h.step(steps)
    b.record(stream)
    h.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    barrier(world)
    return h, {"total_ms": a.elapsed_time(b), "pairs": h.pairs_evaluated() - p0,
               "launches": h.kernel_launches() - l0, "clocks": clk}


def measure_shuffled(pkg, ns, cfg, steps, warmup, world):
    """Plain FP64 RK2 steps (whole-step graph) on the node set permuted by a
    seeded random order: the same physics, every per-node and per-pair
    access in the caller's numbering scattered."""
    perm = np.random.default_rng(7).permutation(ns.n)
    sh = pkg.generators.NodeSet(ns.pos[perm], ns.vel[perm], ns.mass[perm], ns.rho[perm], ns.eps[perm],
                                ns.H[perm], ns.dx)
    h, r = measure_steps_graph(pkg, sh, cfg, pkg.abi.PRECISION_FP64, steps, warmup, world)
    h.close()
    t = allmax(r["total_ms"], world)
    return {"value": allsum(r["pairs"], world) / (t / 1e3), "unit": METRIC, "ms_per_step": t / steps,
            "steps": steps, "workload": "the headline node set in a seeded random order (plain FP64)"}


def measure_eval(h, reps=10):
    """Duration of one evaluateDerivatives (record pack + pair kernel) on the stream."""
    import torch
    stream = torch.cuda.ExternalStream(h.stream())
    h.build_neighbors()
    h.evaluateDerivatives()
    h.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        h.evaluateDerivatives()
    b.record(stream)
    h.synchronize()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def measure_build(h, reps=10):
    """Duration of one ghost + ConnectivityMap build (sphgpu_build_neighbors) on the stream."""
    import torch
    stream = torch.cuda.ExternalStream(h.stream())
    h.build_neighbors()
    h.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        h.build_neighbors()
    b.record(stream)
    h.synchronize()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def measure_e2e(pkg, ns, cfg, steps, warmup):
    """Public API with host buffers: per step one sphgpu_step_rk2_host call
    takes the state host->device from pinned memory, runs one RK2 step and
    brings the new state back device->host into the same arrays."""
    import torch
    n = ns.n

    def pinned(shape):
        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()

    host = {k: pinned(s) for k, s in (("pos", (n, 3)), ("vel", (n, 3)), ("mass", (n,)), ("rho", (n,)),
                                       ("eps", (n,)), ("H", (n, 6)))}
    host["pos"][:] = ns.pos
    host["vel"][:] = ns.vel
    host["mass"][:] = ns.mass
    host["rho"][:] = ns.rho
    host["eps"][:] = ns.eps
    host["H"][:] = ns.H
    h = pkg.SPHHydro(cfg, n=n)
    lib = h.lib

    def P(a):
        return a.ctypes.data_as(ctypes.c_void_p)

    args = [P(host[k]) for k in ("pos", "vel", "mass", "rho", "eps", "H")]
    pkg.abi.check(lib.sphgpu_set_state(h.h, *args), lib)
    h.build_neighbors()
    h.evaluateDerivatives()
    t = ctypes.c_double(0.0)
    dt = ctypes.c_double()
    pairs = 0

    def one_step():
        pkg.abi.check(lib.sphgpu_step_rk2_host(h.h, *args, *args, ctypes.byref(t), ctypes.byref(dt)), lib)
        return h.num_pairs()

    for _ in range(warmup):
        one_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        pairs += one_step()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    nbytes = n * (3 + 3 + 1 + 1 + 1 + 6) * 8
    return {"value": pairs / el, "unit": METRIC, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
            "ms_per_step": 1e3 * el / steps}


ACCURACY_FIELDS = ["delta velocity hydro", "delta specific thermal energy", "delta mass density",
                   "velocity gradient", "new mass density", "new H", "M SPH gradient correction",
                   "max viscous pressure", "weighted neighbor sum", "delta H", "mass second moment",
                   "effective viscous pressure", "viscous work rate", "normalization"]
STATE_FIELDS = ["position", "velocity", "mass density", "specific thermal energy", "H"]


def field_errors(a, b):
    """Errors of `a` against the FP64 `b`: normwise max ||a - b||_inf /
    ||b||_inf, normwise RMS, and a guarded pointwise max: |a_i - b_i| /
    max(|b_i|, rms(b)) per component, which shows large relative errors at
    nodes where the field is small without dividing by the exact zeros."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.abs(a - b)
    bmax = max(float(np.abs(b).max()), 1e-300)
    brms = max(float(np.sqrt(np.mean(b * b))), 1e-300)
    return {"max_rel": float(d.max() / bmax), "rms_rel": float(np.sqrt(np.mean(d * d)) / brms),
            "pointwise_max_rel": float((d / np.maximum(np.abs(b), brms)).max())}


def energy(h):
    c = h.conservation()
    return float(c[6]), float(c[7])


def position_errors(a, b, box):
    """field_errors of positions with each difference taken to the nearest
    periodic image (a node that crossed a periodic plane in one run and not
    in the other is one box length away, not an error)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 3)
    b = np.asarray(b, dtype=np.float64).reshape(-1, 3)
    L = np.asarray(box, dtype=np.float64)
    d = a - b
    d -= L * np.round(d / L)
    return field_errors(b + d, b)


GROWTH_STEPS = (1, 2, 5, 10, 20, 50, 100, 200, 400)
GROWTH_FIELDS = ("velocity", "specific thermal energy", "delta velocity hydro")


def measure_accuracy(pkg, ns, cfg, steps):
    """Mixed form against plain FP64 from the same start.  At t = 0, every
    derivative field's error (field_errors).  Then both forms step together
    for `steps` RK2 steps: the state and the last mid-point derivatives are
    compared at the end, and the errors of velocity, energy and acceleration
    at checkpoints along the way (error_growth), which separates the
    arithmetic error of the first steps from the divergence of two particle
    systems that start a rounding apart (SPH particle noise is chaotic: any
    perturbation grows until it saturates).  Per-step latency of both forms
    (CUDA events recorded just before and after each step call); the total
    energy at the start and the end as compensated sums (hi + lo, two-sum on
    the device) and the relative drift they give."""
    import torch
    abi = pkg.abi
    cf, cm = cfg.copy(), cfg.copy()
    cf.precision = abi.PRECISION_FP64
    cm.precision = abi.PRECISION_MIXED
    hf, hm = pkg.SPHHydro(cf, ns), pkg.SPHHydro(cm, ns)
    for h in (hf, hm):
        h.build_neighbors()
        h.evaluateDerivatives()
    errs0 = {k: field_errors(hm.field(k), hf.field(k)) for k in ACCURACY_FIELDS}
    out = {"field_error_vs_fp64_t0": errs0,
           "max_field_error_t0": max(v["max_rel"] for v in errs0.values()),
           "steps": steps}
    box = [cfg.xmax[a] - cfg.xmin[a] for a in range(3)]
    e0 = {"plain_fp64": energy(hf), "mixed": energy(hm)}
    per = {"plain_fp64": [], "mixed": []}
    growth = []
    ev = {name: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for name in per}
    streams = {"plain_fp64": torch.cuda.ExternalStream(hf.stream()), "mixed": torch.cuda.ExternalStream(hm.stream())}
    for k in range(1, steps + 1):
        for name, h in (("plain_fp64", hf), ("mixed", hm)):
            a, b = ev[name]
            a.record(streams[name])
            h.step(1)
            b.record(streams[name])
            b.synchronize()
            per[name].append(a.elapsed_time(b))
        if k in GROWTH_STEPS:
            g = {"step": k, "time": hf.time}
            for f in GROWTH_FIELDS:
                g[f] = field_errors(hm.field(f), hf.field(f))["max_rel"]
            g["position"] = position_errors(hm.field("position"), hf.field("position"), box)["max_rel"]
            growth.append(g)
    lat, eng = {}, {}
    for name, h in (("plain_fp64", hf), ("mixed", hm)):
        s = sorted(per[name])
        lat[name] = {"p50_ms": s[len(s) // 2], "p99_ms": s[min(len(s) - 1, int(round(0.99 * (len(s) - 1))))],
                     "max_ms": s[-1], "samples": len(s)}
        e1 = energy(h)
        drift = ((e1[0] - e0[name][0]) + (e1[1] - e0[name][1])) / abs(e0[name][0])
        eng[name] = {"e0": e0[name][0], "e0_lo": e0[name][1], "e1": e1[0], "e1_lo": e1[1],
                     "relative_drift": drift, "abs_relative_drift": abs(drift)}
    errs1 = {k: field_errors(hm.field(k), hf.field(k)) for k in STATE_FIELDS[1:] + ACCURACY_FIELDS}
    errs1["position"] = position_errors(hm.field("position"), hf.field("position"), box)
    out["field_error_vs_fp64_after_steps"] = errs1
    out["max_field_error_after_steps"] = max(v["max_rel"] for v in errs1.values())
    out["error_growth"] = growth
    out["step_latency"] = lat
    out["energy"] = eng
    out["energy_drift"] = {k: v["abs_relative_drift"] for k, v in eng.items()}
    out["energy_sum"] = ("double-double (two-sum) total energy on the device: e = e0 + e0_lo; a drift is "
                         "resolved to about 1e-30 relative")
    hf.close()
    hm.close()
    return out


def measure_rate(pkg, ns, cfg, steps, warmup, eval_reps=5):
    """Step rate (pair-interactions/s, ms per step) and the derivative
    evaluation time of one problem."""
    import torch
    h = pkg.SPHHydro(cfg, ns)
    h.build_neighbors()
    h.initialize()
    h.evaluateDerivatives()
    stream = torch.cuda.ExternalStream(h.stream())
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    h.synchronize()
    a.record(stream)
    for _ in range(eval_reps):
        h.evaluateDerivatives()
    b.record(stream)
    h.synchronize()
    eval_ms = a.elapsed_time(b) / eval_reps
    eval_pairs = h.num_pairs()
    for _ in range(warmup):
        h.step(1)
    h.synchronize()
    a.record(stream)
    pairs = 0
    for _ in range(steps):
        h.step(1)
        pairs += h.num_pairs()
    b.record(stream)
    h.synchronize()
    ms = a.elapsed_time(b)
    h.close()
    return {"value": pairs / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / steps,
            "eval_ms": eval_ms, "eval_pair_interactions_per_s": eval_pairs / (eval_ms / 1e3)}


def measure_config_sod(pkg, steps, warmup):
    """Sod tube, plain FP64: 256x32x32 = 262,144 nodes, cubic B-spline
    nPerh 1.51 (~122 neighbors), fixed dt 1e-4."""
    gen, abi = pkg.generators, pkg.abi
    box = ((0.0, 0.0, 0.0), (1.0, 0.125, 0.125))
    ns = gen.sod(nx=256, ny=32, nz=32, box=box)
    out = {}
    for name, prec in (("plain_fp64", abi.PRECISION_FP64), ("mixed", abi.PRECISION_MIXED)):
        out[name] = measure_rate(pkg, ns, gen.sod_config(abi, ns_box=box, precision=prec), steps, warmup)
    out["config"] = {"workload": "Sod tube 256x32x32 = 262,144 nodes in [0,1]x[0,0.125]^2 (periodic), "
                                 "cubic B-spline TableKernel(1000) nPerh 1.51, MG Cl=Cq=1, compatible energy, "
                                 "fixed dt 1e-4"}
    return out


def measure_config_crk(pkg, steps, warmup, drift_steps):
    """CRKSPH Kelvin-Helmholtz 128x128x64 = 1,048,576 nodes (Wendland C4,
    nPerh 1.35, linear corrections, CRKSumVolume): plain FP64 against the
    mixed form, step rate and energy drift over `drift_steps` steps."""
    gen, abi = pkg.generators, pkg.abi
    ns = gen.kelvin_helmholtz(nx=128, ny=128, nz=64, box=((0, 0, 0), (1.0, 1.0, 1.0)))
    relax_h(pkg, ns, gen.kh_config(abi))
    out = {}
    for name, prec in (("plain_fp64", abi.PRECISION_FP64), ("mixed", abi.PRECISION_MIXED)):
        cfg = gen.kh_config(abi, hydro=abi.HYDRO_CRKSPH, precision=prec)
        out[name] = measure_rate(pkg, ns, cfg, steps, warmup)
        if drift_steps > 0:
            h = pkg.SPHHydro(cfg, ns)
            h.build_neighbors()
            h.initialize()
            h.evaluateDerivatives()
            e0 = energy(h)
            h.step(drift_steps)
            e1 = energy(h)
            out[name]["energy_drift"] = abs(((e1[0] - e0[0]) + (e1[1] - e0[1])) / abs(e0[0]))
            out[name]["energy"] = {"e0": e0[0], "e0_lo": e0[1], "e1": e1[0], "e1_lo": e1[1]}
            out[name]["drift_steps"] = drift_steps
            h.close()
    out["mixed_over_plain"] = out["mixed"]["value"] / out["plain_fp64"]["value"]
    out["config"] = {"workload": "CRKSPH Kelvin-Helmholtz 128x128x64 = 1,048,576 nodes in the unit cube "
                                 "(dz = 2 dx), Wendland C4 nPerh 1.35, linear corrections, CRKSumVolume, "
                                 "Courant dt"}
    return out


def batch_specs(pkg, count, precision, seed=20261203, nmin=4096, nmax=262144):
    """The batched-ensemble workload: `count` Sod-type tubes, n log-uniform in
    [nmin, nmax] as an 8k x k x k lattice, gamma ~ U[1.3, 1.67], left/right
    density ratio ~ U[2, 8], cubic B-spline nPerh 1.51."""
    gen, abi = pkg.generators, pkg.abi
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        kk = int(min(32, max(8, round((n / 8.0) ** (1.0 / 3.0)))))
        gamma = float(rng.uniform(1.3, 1.67))
        ratio = float(rng.uniform(2.0, 8.0))
        box = ((0.0, 0.0, 0.0), (1.0, 0.125, 0.125))
        ns = gen.sod(nx=8 * kk, ny=kk, nz=kk, box=box, gamma=gamma, rho1=1.0, rho2=1.0 / ratio, P1=1.0,
                     P2=0.1795, seed=seed + 1 + k)
        cfg = gen.sod_config(abi, ns_box=box, gamma=gamma, precision=precision)
        out.append((ns, cfg))
    return out


def time_batch(pkg, probs, steps, warmup, world, graph):
    """K batched steps of `probs` in one call (autotuned schedules; the whole
    RK2 step replayed as a captured CUDA graph when `graph`, eager launches
    otherwise), timed with CUDA events on the batch stream, max over ranks;
    pairs from the device-side pair counter."""
    import torch
    batch = pkg.SPHBatch(probs)
    batch.build_neighbors()
    batch.evaluateDerivatives()
    tune = batch.autotune()
    batch.set_schedule("step graph", 1 if graph else 0)
    stream = torch.cuda.ExternalStream(batch.stream())
    for _ in range(warmup):
        batch.step(1)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = batch.kernel_launches()
    p0 = batch.pairs_evaluated()
    e0.record(stream)
    batch.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    t = allmax(e0.elapsed_time(e1) / 1e3, world)
    pairs = allsum(batch.pairs_evaluated() - p0, world)
    launches = batch.kernel_launches() - l0
    batch.close()
    return {"value": pairs / t, "unit": METRIC, "ms_per_step": 1e3 * t / steps,
            "kernel_launches_per_step": launches / steps, "step_graph": bool(graph),
            "autotuned": {"neighbor walk": ["auto", "thread per node", "warp per node"][tune["neighbor walk"]],
                          "neighbor cells per kernel reach": tune["neighbor cells"],
                          "pair loop threads": tune["pair loop"]}}


def measure_batch(pkg, count, steps, warmup, rank=0, world=1):
    """Batched ensemble, mixed form: every stage one launch over all members,
    the whole RK2 step replayed as a captured CUDA graph;
    against the same batch in plain FP64, and against the mixed problems
    stepped one at a time (one launch sequence per problem).  With N GPUs the
    tubes are placed by size (longest first onto the least-loaded rank; no
    exchange on the data path); the lines take the max time over ranks and the
    sum of the pairs."""
    import torch
    abi = pkg.abi
    out = {}
    nodes = None
    for name, prec in (("mixed", abi.PRECISION_MIXED), ("plain_fp64", abi.PRECISION_FP64)):
        specs = batch_specs(pkg, count, prec)
        place = pkg.sharding.partition_by_cost([ns.n for ns, _ in specs], world)
        mine = pkg.sharding.local_items(place, rank)
        specs = [specs[k] for k in mine]
        nodes = allsum(sum(ns.n for ns, _ in specs), world)
        probs = [pkg.SPHHydro(cfg, ns) for ns, cfg in specs]
        out[name] = time_batch(pkg, probs, steps, warmup, world, graph=True)
        if name == "mixed":
            out["mixed_eager"] = time_batch(pkg, probs, steps, warmup, world, graph=False)
            # one launch sequence per problem: host clock around device synchronisation
            for _ in range(warmup):
                for p in probs:
                    p.step(1)
            torch.cuda.synchronize()
            barrier(world)
            t0 = time.perf_counter()
            lpairs = 0
            for _ in range(steps):
                for p in probs:
                    p.step(1)
                    lpairs += p.num_pairs()
            torch.cuda.synchronize()
            t_loop = allmax(time.perf_counter() - t0, world)
            lpairs = allsum(lpairs, world)
            out["one_launch_per_problem"] = {"value": lpairs / t_loop, "unit": METRIC,
                                             "ms_per_step": 1e3 * t_loop / steps}
        for p in probs:
            p.close()
    out["value"] = out["mixed"]["value"]
    out["unit"] = METRIC
    out["mixed_over_plain"] = out["mixed"]["value"] / out["plain_fp64"]["value"]
    out["batched_over_loop"] = out["mixed"]["value"] / out["one_launch_per_problem"]["value"]
    out["config"] = {"workload": "%d Sod-type tubes, n log-uniform in [4096, 262144] (8k x k x k), "
                                 "gamma ~ U[1.3, 1.67], density ratio ~ U[2, 8], cubic B-spline nPerh 1.51, "
                                 "fixed dt 1e-4" % count,
                     "nodes": nodes, "steps": steps, "warmup": warmup,
                     "placement": "tubes placed on %d GPU(s) by size, no data-path exchange" % world}
    return out


def measure_serving(pkg, duration, nsteps, rate=20.0, budget=150e9, rank=0, world=1):
    """Continuous-batching request loop on a seeded Poisson trace, mixed form
    and plain FP64 on the same trace.  With N GPUs every rank routes the
    trace identically (least outstanding estimated work at arrival) and
    serves its share; times to completion and pairs are gathered to rank 0."""
    s = pkg.serving
    trace = s.poisson_trace(rate=rate, duration=duration, nsteps=nsteps)
    route = pkg.sharding.route_requests([r["arrival"] for r in trace],
                                        [r["n"] * r["nsteps"] * 1.0e-8 for r in trace], world)
    mine = [trace[k] for k in pkg.sharding.local_items(route, rank)]
    out = {}
    for name, prec in (("mixed", pkg.abi.PRECISION_MIXED), ("plain_fp64", pkg.abi.PRECISION_FP64)):
        # untimed warm-up on the first requests (library, allocator pool)
        if mine:
            s.serve(mine[:4], prec, budget_bytes=budget)
        barrier(world)
        ttc, makespan, stats = s.serve(mine, prec, budget_bytes=budget) if mine else ([], 0.0, None)
        local = {"ttc": ttc, "makespan": makespan,
                 "pairs": stats["pair_interactions"] if stats else 0.0,
                 "completed": int(stats["completed"]) if stats else 0,
                 "peak": stats["peak_bytes"] if stats else 0.0,
                 "ticks": int(stats["ticks"]) if stats else 0}
        parts = [local]
        if world > 1:
            import torch.distributed as dist
            parts = [None] * world
            dist.all_gather_object(parts, local)
        t = np.array([x for p in parts for x in p["ttc"]])
        span = max(p["makespan"] for p in parts)
        out[name] = {"ttc_p50_s": float(np.percentile(t, 50)), "ttc_p99_s": float(np.percentile(t, 99)),
                     "pair_interactions_per_s": sum(p["pairs"] for p in parts) / span, "makespan_s": span,
                     "completed": sum(p["completed"] for p in parts),
                     "peak_device_gb": max(p["peak"] for p in parts) / 1e9,
                     "batched_steps": sum(p["ticks"] for p in parts)}
    out["config"] = {"trace": "Poisson arrivals at %.0f/s for %.1f s (%d requests, seeded), 50/50 "
                              "Kelvin-Helmholtz / Sod-type, n log-uniform in [8192, 1048576], %d RK2 steps each, "
                              "admission by device footprint under %.0f GB per GPU, routed to %d GPU(s)"
                              % (rate, duration, len(trace), nsteps, budget / 1e9, world)}
    if duration < 60.0 or nsteps < 200:
        out["config"]["shortened"] = (
            "SHORTENED trace: %.1f s of arrivals and %d steps per request instead of the specified 60 s and 200 "
            "steps; the specified trace holds about 8 minutes of GPU work per form, beyond the bench's time "
            "limit (bench.py --serving 60 --serving-steps 200 runs it)" % (duration, nsteps))
    return out


REF_SPH = os.path.join(ROOT, "oracle", "_ref", "ref_sph")


def write_reference_input(path, cfg, ns, nsteps):
    """Input of oracle/_ref/ref_sph: int64 n, int64 steps, the raw
    sphgpu_config, then the node arrays in the reference Field layouts."""
    with open(path, "wb") as f:
        f.write(np.int64(ns.n).tobytes())
        f.write(np.int64(nsteps).tobytes())
        f.write(bytes(cfg))
        for a in (ns.pos, ns.vel, ns.mass, ns.rho, ns.eps, ns.H):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())


def time_reference(cfg, ns, steps, warmup):
    """The reference's own SPHHydroBase + CheapSynchronousRK2 (compiled from
    its sources into oracle/_ref/ref_sph): seconds and pair interactions of
    `steps` timed RK2 steps after `warmup` untimed ones, one core; H relaxed
    by the reference's own iterateIdealH first (untimed)."""
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "in.bin")
        write_reference_input(path, cfg, ns, steps)
        out = subprocess.check_output([REF_SPH, "--time", str(warmup), path,
                                       str(IDEAL_H[0]), repr(IDEAL_H[1])]).decode()
    r = json.loads(out.strip().splitlines()[-1])
    return r["seconds"], r["pairs"]


def cpu_baseline(pkg, nx):
    """The reference's CPU path on the host, one core, on a bounded sample of
    the workload: a z-slab of the same lattice (same spacing, stencil and
    state), two timed RK2 steps after one untimed.  Falls back to the oracle
    (the FP64 restatement of the reference path) where the reference could
    not be compiled."""
    nz = max(4, nx // 8)
    ns, cfg = kh_problem(pkg, nx, nz)
    if os.path.exists(REF_SPH):
        el, pairs = time_reference(cfg, ns, 2, 1)
        kind, what = "reference", "the reference's own SPHHydroBase + CheapSynchronousRK2 (oracle/_ref/ref_sph)"
    else:
        import oracle
        o = oracle.OracleProblem(cfg, ns)
        o.iterate_ideal_h(*IDEAL_H)
        o.build_neighbors()
        o.evaluate_derivatives()
        o.step(1)
        t0 = time.perf_counter()
        o.step(2)
        el = time.perf_counter() - t0
        pairs = 2 * o.num_pairs()
        kind, what = "port", "the oracle restatement of the reference path"
    return {"value": pairs / el, "unit": METRIC, "cores": 1, "kind": kind,
            "sample": "%s, serial, on a %dx%dx%d z-slab of the lattice (%d nodes, same spacing and stencil), "
                      "2 timed RK2 steps, %.1f s" % (what, nx, nx, nz, ns.n, el),
            "cpu": platform.processor() or platform.machine()}


# ------------------------------------------------------------------ reference arm
def _ref_worker(args):
    idx, nx, nz, steps, warmup, barrier_obj, q = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        os.sched_setaffinity(0, {idx % os.cpu_count()})
    except Exception:
        pass
    pkg = importlib.import_module("llnl-spheral_b200")
    ns, cfg = kh_problem(pkg, nx, nz, seed=20261203 + idx)
    barrier_obj.wait()
    if os.path.exists(REF_SPH):
        el, pairs = time_reference(cfg, ns, steps, warmup)
    else:
        import oracle
        o = oracle.OracleProblem(cfg, ns)
        o.iterate_ideal_h(*IDEAL_H)
        o.build_neighbors()
        o.evaluate_derivatives()
        for _ in range(warmup):
            o.step(1)
        t0 = time.perf_counter()
        pairs = 0
        for _ in range(steps):
            o.step(1)
            pairs += o.num_pairs()
        el = time.perf_counter() - t0
    q.put((pairs, el))


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = max(1, min(os.cpu_count() or 1, 32))
    try:
        import psutil
        # each process holds about 0.8 GB for a 128x128x16 slab
        cores = max(1, min(cores, int(psutil.virtual_memory().available / 2.0e9)))
    except Exception:
        pass
    nx = args.nx
    # bounded sample per process: a z-slab of the same lattice (same dx, same
    # stencil); thinner when many steps are asked for
    total = args.steps + args.warmup
    nz = max(4, nx // 8 if total <= 16 else nx // 16 if total <= 64 else nx // 32)
    ctx = mp.get_context("spawn")
    bar = ctx.Barrier(cores)
    q = ctx.Queue()
    procs = [ctx.Process(target=_ref_worker, args=((i, nx, nz, args.steps, args.warmup, bar, q),))
             for i in range(cores)]
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    pairs = sum(r[0] for r in res)
    el = max(r[1] for r in res)
    value = pairs / el
    kind = "reference" if os.path.exists(REF_SPH) else "port"
    what = ("the reference's own SPHHydroBase + CheapSynchronousRK2 compiled from its sources (oracle/_ref/ref_sph)"
            if kind == "reference" else "the oracle restatement of the reference FP64 path")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": bench_config(args.nx),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind,
                             "sample": "%s, one serial process per core, each a %dx%dx%d z-slab of the lattice "
                                       "(same spacing, stencil and state), %d timed RK2 steps after %d untimed"
                                       % (what, nx, nx, nz, args.steps, args.warmup)},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def bench_config(nx):
    """The `config` both arms print (the same workload, the same precision)."""
    return {"workload": WORKLOAD, "nodes": nx * nx * nx, "precision": "FP64 (the reference's arithmetic)"}


# ------------------------------------------------------------------ our arm
def run_ours(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    pkg = importlib.import_module("llnl-spheral_b200")
    importlib.import_module("llnl-spheral_b200.build").build()
    abi = pkg.abi
    ns, cfg = kh_problem(pkg, args.nx, seed=20261203 + rank)
    relax_h(pkg, ns, cfg)
    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    clocks = Clocks(vis[local] if local < len(vis) else local)
    # headline: plain FP64, the reference's precision; K steps in one
    # sphgpu_step_rk2 call (the captured whole-step graph replayed K times)
    hg, rp = measure_steps_graph(pkg, ns, cfg, abi.PRECISION_FP64, args.steps, args.warmup, world, clocks)
    hg.close()
    t_plain = allmax(rp["total_ms"], world)
    pairs_plain = allsum(rp["pairs"], world)
    # the mixed FP32-pair form on the same workload
    hg, rm = measure_steps_graph(pkg, ns, cfg, abi.PRECISION_MIXED, args.steps, args.warmup, world)
    hg.close()
    del hg
    t_mixed = allmax(rm["total_ms"], world)
    pairs_mixed = allsum(rm["pairs"], world)
    value = pairs_plain / (t_plain / 1e3)
    mixed_value = pairs_mixed / (t_mixed / 1e3)
    # one call per step (per-step latency), graph replays and eager launches
    hp, lp = measure_steps(pkg, ns, cfg, abi.PRECISION_FP64, args.steps, args.warmup, world)
    hm, lm = measure_steps(pkg, ns, cfg, abi.PRECISION_MIXED, args.steps, args.warmup, world)
    per_call = {}
    for form, prec, r in (("fp64", abi.PRECISION_FP64, lp), ("mixed", abi.PRECISION_MIXED, lm)):
        he, re_ = measure_steps(pkg, ns, cfg, prec, args.steps, args.warmup, world, graph=False)
        he.close()
        del he
        tl = allmax(r["total_ms"], world)
        te = allmax(re_["total_ms"], world)
        per_call[form] = {"graph_replay": {"value": allsum(r["pairs"], world) / (tl / 1e3),
                                           "ms_per_step": tl / args.steps},
                          "eager": {"value": allsum(re_["pairs"], world) / (te / 1e3),
                                    "ms_per_step": te / args.steps, "gpu_launches": re_["launches"]}}
    # roofline of the dominant kernel pair of the step (evaluateDerivatives:
    # record pack + pair kernel), each form
    peak, peak_kind = load_peaks()
    g = ctypes.c_int64()
    e = ctypes.c_int64()
    hp.lib.sphgpu_connectivity_size(hp.h, ctypes.byref(g), ctypes.byref(e))
    nodes, ghosts, entries = ns.n, g.value, e.value
    t_eval_plain = measure_eval(hp)
    t_eval_mixed = measure_eval(hm)
    t_build_plain = measure_build(hp)
    t_build_mixed = measure_build(hm)

    def roofline(form, alg, t_eval, kernel):
        achieved = alg / (t_eval / 1e3) / 1e9
        measured = EVAL_TRAFFIC_96[form]
        units96 = eval_alg_bytes_fp64(*EVAL_UNITS_96) if form == "fp64" else eval_alg_bytes_mixed(*EVAL_UNITS_96)
        return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind + " (MEASURED_PEAKS hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "unit": "GB/s", "frac": achieved / peak,
                "traffic": None if measured is None else measured * alg / units96,
                "traffic_source": None if measured is None else
                "ncu dram__bytes_read.sum + dram__bytes_write.sum of the two kernels on Kelvin-Helmholtz 96^3, "
                "scaled by the algorithmic bytes",
                "algorithmic_bytes": alg, "eval_ms": t_eval}

    result = None
    if rank == 0:
        def pct(v, q):
            v = sorted(v)
            return v[min(len(v) - 1, int(round(q * (len(v) - 1))))]
        result = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_plain / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args.nx),
            "timing": "K steps in one sphgpu_step_rk2 call (whole-step CUDA graph replayed K times, no "
                      "host synchronisation between steps), CUDA events on the problem's stream",
            "problem": {"nodes_per_gpu": nodes, "ghosts": ghosts, "pairs_per_step": rp["pairs"] / args.steps,
                        "parallelism": "one independent problem per GPU" if world > 1 else "single GPU",
                        "l2": "inputs larger than L2 (state %.2f GB, pair records %.2f GB)" % (
                            nodes * 18 * 8 / 1e9, (nodes + ghosts) * 160 / 1e9)},
            "latency_ms": {"p50": pct(lp["per_step_ms"], 0.5), "p99": pct(lp["per_step_ms"], 0.99),
                           "of": "one sphgpu_step_rk2 call per step"},
            "stage_ms": {"neighbor_build": t_build_plain, "evaluate_derivatives": t_eval_plain,
                         "rk2_step": t_plain / args.steps},
            "mixed": {"value": mixed_value, "unit": METRIC, "ms_per_step": t_mixed / args.steps,
                      "dtype": "f32 pair / f64 state",
                      "latency_ms": {"p50": pct(lm["per_step_ms"], 0.5), "p99": pct(lm["per_step_ms"], 0.99)},
                      "stage_ms": {"neighbor_build": t_build_mixed, "evaluate_derivatives": t_eval_mixed,
                                   "rk2_step": t_mixed / args.steps},
                      "roofline": roofline("mixed", eval_alg_bytes_mixed(nodes, ghosts, entries), t_eval_mixed,
                                           "evaluateDerivatives (pack_mixed + sph_eval_mixed)"),
                      "gpu_launches": rm["launches"]},
            "mixed_over_plain": mixed_value / value,
            "one_call_per_step": per_call,
            "roofline": roofline("fp64", eval_alg_bytes_fp64(nodes, ghosts, entries), t_eval_plain,
                                 "evaluateDerivatives (pack_records + sph_eval_fp64)"),
            "gpu_launches": rp["launches"],
            "clocks": rp["clocks"],
        }
        if not args.no_e2e:
            esteps = max(3, args.steps // 2)
            result["e2e"] = measure_e2e(pkg, ns, cfg, esteps, 1)
            cm = cfg.copy()
            cm.precision = abi.PRECISION_MIXED
            result["mixed"]["e2e"] = measure_e2e(pkg, ns, cm, esteps, 1)
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(pkg, args.nx)
    hm.close()
    hp.close()
    # the same node set in a seeded random order: nothing reorders the
    # caller's nodes, so the pair kernels' gathers follow the caller's order
    shuffled = measure_shuffled(pkg, ns, cfg, max(3, args.steps // 5), args.warmup, world)
    if rank == 0:
        result["shuffled_input"] = shuffled
    if args.accuracy_steps > 0:
        acc = measure_accuracy(pkg, ns, cfg, args.accuracy_steps)
        if rank == 0:
            result["accuracy"] = acc
    if args.configs:
        rsod = measure_config_sod(pkg, max(3, args.steps // 2), 2)
        rcrk = measure_config_crk(pkg, max(3, args.steps // 2), 2, args.accuracy_steps)
        if rank == 0:
            result["sod_fp64"] = rsod
            result["crk_kh"] = rcrk
    if args.batch > 0:
        rb = measure_batch(pkg, args.batch, max(2, args.steps // 3), 1, rank, world)
        if rank == 0:
            result["batch"] = rb
    if args.serving > 0:
        rs = measure_serving(pkg, args.serving, args.serving_steps, rank=rank, world=world)
        if rank == 0:
            result["serving"] = rs
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)
    return 0


def kernel_survey():
    """Kelvin-Helmholtz 96^3 (SPH, mixed then FP64) and CRKSPH
    Kelvin-Helmholtz 64x64x32 (mixed then FP64): build, initialize, one
    derivative evaluation and two RK2 steps each, so that every kernel of
    the path launches; nothing is timed."""
    pkg = importlib.import_module("llnl-spheral_b200")
    abi, gen = pkg.abi, pkg.generators
    ns, cfg = kh_problem(pkg, 96)
    ns2 = gen.kelvin_helmholtz(nx=64, ny=64, nz=32, box=((0, 0, 0), (1.0, 1.0, 1.0)))
    cases = [(ns, cfg, prec) for prec in (abi.PRECISION_MIXED, abi.PRECISION_FP64)]
    cases += [(ns2, gen.kh_config(abi, hydro=abi.HYDRO_CRKSPH, precision=prec), None)
              for prec in (abi.PRECISION_MIXED, abi.PRECISION_FP64)]
    for nodes, c, prec in cases:
        if prec is not None:
            c = c.copy()
            c.precision = prec
        h = pkg.SPHHydro(c, nodes)
        h.build_neighbors()
        h.initialize()
        h.evaluateDerivatives()
        h.step(2)
        h.synchronize()
        h.close()
    print(json.dumps({"kernel_survey": "done", "problems": len(cases)}))
    return 0


def main():
    args = parse()
    if args.kernel_survey:
        return kernel_survey()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
