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
mixed FP32-pair form; the plain FP64 form and p50/p99 step latency are in
the same line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import importlib
import json
import multiprocessing as mp
import os
import platform
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
            "RigorousSumDensity, IdealH, Courant dt (cfl 0.25); one CheapSynchronousRK2 step per step")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=128, help="lattice size per axis (default: the full workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def kh_problem(pkg, nx, nz=None, seed=20261203):
    gen, abi = pkg.generators, pkg.abi
    nz = nz or nx
    ns = gen.kelvin_helmholtz(nx=nx, ny=nx, nz=nz, box=((0, 0, 0), (1.0, 1.0, nz / nx)), seed=seed)
    cfg = gen.kh_config(abi, xmax=(1.0, 1.0, nz / nx))
    return ns, cfg


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
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
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


def measure_steps(pkg, ns, cfg, precision, steps, warmup, world, clocks=None):
    import torch
    c = cfg.copy()
    c.precision = precision
    h = pkg.SPHHydro(c, ns)
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


def measure_e2e(pkg, ns, cfg, steps, warmup):
    """Public API with host buffers: per step the state goes host->device
    (sphgpu_set_state from pinned memory), one RK2 step runs, and the new
    state comes back device->host (sphgpu_get_state)."""
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
        pkg.abi.check(lib.sphgpu_set_state(h.h, *args), lib)
        pkg.abi.check(lib.sphgpu_step_rk2(h.h, ctypes.byref(t), 1, ctypes.byref(dt)), lib)
        pkg.abi.check(lib.sphgpu_get_state(h.h, *args), lib)
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


def cpu_baseline(pkg, ns, cfg):
    """The oracle (a serial FP64 restatement of the reference path) on the
    same workload: one RK2 step after the start-up evaluation, 1 core."""
    import oracle
    o = oracle.OracleProblem(cfg, ns)
    o.build_neighbors()
    o.evaluate_derivatives()
    t0 = time.perf_counter()
    o.step(1)
    el = time.perf_counter() - t0
    pairs = o.num_pairs()
    return {"value": pairs / el, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": "1 CheapSynchronousRK2 step of the full %d-node workload (ghosts, neighbors, "
                      "derivatives, updates), serial oracle, %.1f s" % (ns.n, el),
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
    import oracle
    ns, cfg = kh_problem(pkg, nx, nz, seed=20261203 + idx)
    o = oracle.OracleProblem(cfg, ns)
    o.build_neighbors()
    o.evaluate_derivatives()
    for _ in range(warmup):
        o.step(1)
    barrier_obj.wait()
    t0 = time.perf_counter()
    pairs = 0
    for _ in range(steps):
        o.step(1)
        pairs += o.num_pairs()
    q.put((pairs, time.perf_counter() - t0))


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    oracle.lib()
    cores = max(1, min(os.cpu_count() or 1, 32))
    try:
        import psutil
        cores = max(1, min(cores, int(psutil.virtual_memory().available / 1.0e9)))
    except Exception:
        pass
    nx = args.nx
    nz = max(4, nx // 8)          # bounded sample: a z-slab of the same lattice (same dx, same stencil)
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
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_nodes_per_process": nx * nx * nz,
                       "sample": "%d concurrent processes, each a %dx%dx%d z-slab of the lattice "
                                 "(same spacing and stencil), %d RK2 steps" % (cores, nx, nx, nz, args.steps)},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port",
                             "sample": "oracle restatement of the reference FP64 path, one serial process per core"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
def run_ours(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    pkg = importlib.import_module("llnl-spheral_b200")
    importlib.import_module("llnl-spheral_b200.build").build()
    abi = pkg.abi
    ns, cfg = kh_problem(pkg, args.nx, seed=20261203 + rank)
    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    clocks = Clocks(vis[local] if local < len(vis) else local)
    # headline: mixed form
    hm, rm = measure_steps(pkg, ns, cfg, abi.PRECISION_MIXED, args.steps, args.warmup, world, clocks)
    t_mixed = allmax(rm["total_ms"], world)
    pairs_mixed = allsum(rm["pairs"], world)
    # plain FP64 on the same workload
    hp, rp = measure_steps(pkg, ns, cfg, abi.PRECISION_FP64, args.steps, args.warmup, world)
    t_plain = allmax(rp["total_ms"], world)
    pairs_plain = allsum(rp["pairs"], world)
    value = pairs_mixed / (t_mixed / 1e3)
    plain_value = pairs_plain / (t_plain / 1e3)
    # roofline of the dominant kernel (derivative evaluation)
    peak, peak_kind = load_peaks()
    g = ctypes.c_int64()
    e = ctypes.c_int64()
    hm.lib.sphgpu_connectivity_size(hm.h, ctypes.byref(g), ctypes.byref(e))
    t_eval_mixed = measure_eval(hm)
    t_eval_plain = measure_eval(hp)
    nodes, ghosts, entries = ns.n, g.value, e.value
    alg_bytes = (nodes + ghosts) * 152 + nodes * 576 + 4 * entries
    achieved = alg_bytes / (t_eval_mixed / 1e3) / 1e9
    result = None
    if rank == 0:
        lat = sorted(rm["per_step_ms"])
        latp = sorted(rp["per_step_ms"])

        def pct(v, q):
            return v[min(len(v) - 1, int(round(q * (len(v) - 1))))]
        result = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mixed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair / f64 state", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nodes_per_gpu": nodes, "ghosts": ghosts,
                       "pairs_per_step": rm["pairs"] / args.steps, "precision": "mixed FP32-pair/FP64-critical",
                       "parallelism": "one independent problem per GPU" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (state %.2f GB, pair records %.2f GB)" % (
                           nodes * 18 * 8 / 1e9, (nodes + ghosts) * 160 / 1e9)},
            "latency_ms": {"p50": pct(lat, 0.5), "p99": pct(lat, 0.99)},
            "plain_fp64": {"value": plain_value, "unit": METRIC, "ms_per_step": t_plain / args.steps,
                           "latency_ms": {"p50": pct(latp, 0.5), "p99": pct(latp, 0.99)},
                           "eval_ms": t_eval_plain},
            "mixed_over_plain": value / plain_value,
            "roofline": {"bound": "hbm", "kernel": "evaluateDerivatives (record pack + sph_eval_mixed)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "algorithmic_bytes": alg_bytes, "eval_ms": t_eval_mixed},
            "gpu_launches": rm["launches"],
            "clocks": rm["clocks"],
        }
        if not args.no_e2e:
            cm = cfg.copy()
            cm.precision = abi.PRECISION_MIXED
            result["e2e"] = measure_e2e(pkg, ns, cm, max(3, args.steps // 2), 1)
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(pkg, ns, cfg)
    hm.close()
    hp.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
