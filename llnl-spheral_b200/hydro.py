"""Host-side mirror of the reference's hydro package interface over the C-ABI.

``SPHHydro`` keeps the names and argument meaning of Spheral's SPH factory
(src/SPH/SPHHydros.py:12-59) and of the Physics<Dim> methods the integrator
calls (src/Physics/Physics.hh:51-159): ``initialize``, ``evaluateDerivatives``,
``finalizeDerivatives``, ``finalize``, ``dt``; fields are read by the
reference's State/StateDerivatives keys (src/Hydro/HydroFieldNames.cc).
``CheapSynchronousRK2Integrator.step`` advances one
CheapSynchronousRK2::step (src/Integrator/CheapSynchronousRK2.cc:81-143).

Every call goes through libsphgpu.so; errors raise RuntimeError with the
library's message (the reference throws VERIFYError).  There is no CPU path.
"""
import ctypes
import os

import numpy as np

from . import abi

FIELD_COMPONENTS = {
    "position": 3, "velocity": 3, "mass": 1, "mass density": 1, "specific thermal energy": 1, "H": 6,
    "pressure": 1, "sound speed": 1, "grad h corrections": 1, "new mass density": 1, "normalization": 1,
    "delta position": 3, "delta mass density": 1, "delta velocity hydro": 3,
    "delta specific thermal energy": 1, "velocity gradient": 9, "internal velocity gradient": 9,
    "M SPH gradient correction": 9, "local M SPH gradient correction": 9, "delta H": 6, "new H": 6,
    "max viscous pressure": 1, "effective viscous pressure": 1, "viscous work rate": 1,
    "XSPH weight sum": 1, "XSPH delta vi": 3, "weighted neighbor sum": 1, "mass second moment": 6,
    "node volume": 1, "A CRKSPH correction": 1, "B CRKSPH correction": 3, "grad A CRKSPH correction": 3,
    "grad B CRKSPH correction": 9, "m0 CRKSPH moment": 1, "m1 CRKSPH moment": 3, "m2 CRKSPH moment": 6,
    "grad m0 CRKSPH moment": 3, "grad m1 CRKSPH moment": 9, "grad m2 CRKSPH moment": 27,
    "mass density gradient": 3,
}


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _tune_report(out):
    best = min(out[1], out[2])
    return {"neighbor walk": int(out[0]), "neighbor walk ms": {"thread": out[1], "warp": out[2]},
            "neighbor cells": int(out[6]), "neighbor cells ms": {1: best, 2: out[7]},
            "pair loop": int(out[3]), "pair loop ms": {64: out[4], 128: out[5]}}


class SPHHydro:
    """One FluidNodeList evolved by the B200 SPH hydro path.

    ``cfg`` is an ``abi.SphConfig`` (see ``abi.make_config``); ``nodes`` a
    ``generators.NodeSet`` (or anything with pos, vel, mass, rho, eps, H AoS
    arrays).
    """

    def __init__(self, cfg, nodes=None, n=None):
        self.lib = abi.load_library()
        self.cfg = cfg.copy()
        self.n = int(nodes.n if nodes is not None else n)
        h = ctypes.c_void_p()
        abi.check(self.lib.sphgpu_create(ctypes.byref(self.cfg), self.n, ctypes.byref(h)), self.lib)
        self.h = h
        self.time = 0.0
        if nodes is not None:
            self.set_state(nodes)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.sphgpu_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state
    def set_state(self, nodes):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (nodes.pos, nodes.vel, nodes.mass, nodes.rho, nodes.eps, nodes.H)]
        abi.check(self.lib.sphgpu_set_state(self.h, *[_p(a) for a in arrs]), self.lib)

    def set_state_device(self, ptrs):
        """ptrs: six device pointers (int) in the order of set_state."""
        abi.check(self.lib.sphgpu_set_state_device(self.h, *[ctypes.c_void_p(int(q)) for q in ptrs]), self.lib)

    def field(self, key):
        c = FIELD_COMPONENTS[key]
        out = np.empty(self.n * c)
        abi.check(self.lib.sphgpu_get_field(self.h, key.encode(), _p(out), out.size), self.lib)
        return out.reshape(self.n, c) if c > 1 else out

    def set_field(self, key, values):
        """Write a State / StateDerivatives field by its key (n x components)."""
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        abi.check(self.lib.sphgpu_set_field(self.h, key.encode(), _p(v), v.size), self.lib)

    def set_dt_bounds(self, dt_min, dt_max):
        abi.check(self.lib.sphgpu_set_dt_bounds(self.h, float(dt_min), float(dt_max)), self.lib)

    # ---- Integrator::setGhostNodes + ConnectivityMap
    def build_neighbors(self):
        abi.check(self.lib.sphgpu_build_neighbors(self.h), self.lib)

    setGhostNodes = build_neighbors

    def connectivity(self):
        g = ctypes.c_int64()
        e = ctypes.c_int64()
        abi.check(self.lib.sphgpu_connectivity_size(self.h, ctypes.byref(g), ctypes.byref(e)), self.lib)
        off = np.empty(self.n + 1, dtype=np.int64)
        nb = np.empty(max(e.value, 1), dtype=np.int32)
        root = np.empty(max(g.value, 1), dtype=np.int32)
        abi.check(self.lib.sphgpu_get_connectivity(self.h, _p(off), _p(nb), _p(root)), self.lib)
        return off, nb[:e.value], root[:g.value]

    def pair_accelerations(self):
        """The reference's pair-wise accelerations of the last evaluation, one
        row per ConnectivityMap entry in row order, (E, 3)
        (sphgpu_get_pair_accelerations)."""
        g = ctypes.c_int64()
        e = ctypes.c_int64()
        abi.check(self.lib.sphgpu_connectivity_size(self.h, ctypes.byref(g), ctypes.byref(e)), self.lib)
        out = np.empty((max(e.value, 1), 3))
        abi.check(self.lib.sphgpu_get_pair_accelerations(self.h, _p(out), 3 * e.value), self.lib)
        return out[:e.value]

    def ghost_positions(self):
        """Ghost node positions of the current connectivity, (G, 3)."""
        g = ctypes.c_int64()
        e = ctypes.c_int64()
        abi.check(self.lib.sphgpu_connectivity_size(self.h, ctypes.byref(g), ctypes.byref(e)), self.lib)
        out = np.empty((max(g.value, 1), 3))
        abi.check(self.lib.sphgpu_get_ghost_positions(self.h, _p(out)), self.lib)
        return out[:g.value]

    def num_pairs(self):
        v = ctypes.c_int64()
        abi.check(self.lib.sphgpu_num_pairs(self.h, ctypes.byref(v)), self.lib)
        return v.value

    def pairs_evaluated(self):
        """num_pairs() of every RK2 step taken so far, summed."""
        v = ctypes.c_int64()
        abi.check(self.lib.sphgpu_pairs_evaluated(self.h, ctypes.byref(v)), self.lib)
        return v.value

    # ---- Physics<Dim> methods
    def initialize(self, time=0.0, dt=0.0):
        abi.check(self.lib.sphgpu_initialize(self.h, time, dt), self.lib)

    def evaluateDerivatives(self, time=0.0, dt=0.0):
        abi.check(self.lib.sphgpu_evaluate_derivatives(self.h, time, dt), self.lib)

    def finalizeDerivatives(self, time=0.0, dt=0.0):
        abi.check(self.lib.sphgpu_finalize_derivatives(self.h, time, dt), self.lib)

    def finalize(self, time=0.0, dt=0.0):
        abi.check(self.lib.sphgpu_finalize(self.h, time, dt), self.lib)

    def dt(self):
        v = ctypes.c_double()
        abi.check(self.lib.sphgpu_dt(self.h, ctypes.byref(v)), self.lib)
        return v.value

    # ---- integrator
    def step(self, nsteps=1):
        t = ctypes.c_double(self.time)
        dt = ctypes.c_double()
        abi.check(self.lib.sphgpu_step_rk2(self.h, ctypes.byref(t), int(nsteps), ctypes.byref(dt)), self.lib)
        self.time = t.value
        return t.value, dt.value

    def step_host(self, state_in, state_out=None):
        """One RK2 step of a host-resident state (sphgpu_step_rk2_host):
        state_in holds the six arrays of set_state (float64, C order),
        state_out six arrays that receive the new state (None: state_in)."""
        state_out = state_in if state_out is None else state_out
        for a in list(state_in) + list(state_out):
            if a is not None and (a.dtype != np.float64 or not a.flags.c_contiguous):
                raise ValueError("step_host arrays must be C-contiguous float64")
        t = ctypes.c_double(self.time)
        dt = ctypes.c_double()
        ptrs = [_p(a) for a in state_in] + [None if a is None else _p(a) for a in state_out]
        abi.check(self.lib.sphgpu_step_rk2_host(self.h, *ptrs, ctypes.byref(t), ctypes.byref(dt)), self.lib)
        self.time = t.value
        return t.value, dt.value

    def conservation(self):
        out = np.empty(8)
        abi.check(self.lib.sphgpu_conservation(self.h, _p(out)), self.lib)
        return out

    def iterateIdealH(self, maxIdealHIterations=50, idealHTolerance=1.0e-4):
        """SpheralController.iterateIdealH: relax H to the ideal smoothing
        scale before the run.  Returns (iterations, last max change of H)."""
        itr = ctypes.c_int32()
        dh = ctypes.c_double()
        abi.check(self.lib.sphgpu_iterate_ideal_h(self.h, int(maxIdealHIterations), float(idealHTolerance),
                                                  ctypes.byref(itr), ctypes.byref(dh)), self.lib)
        return itr.value, dh.value

    def checkpoint(self):
        """Checkpoint image (bytes) of the state, derivatives, time, last dt
        and cycle: SPHHydroBase::dumpState plus the NodeList and integrator
        state."""
        size = ctypes.c_int64()
        abi.check(self.lib.sphgpu_checkpoint_size(self.h, ctypes.byref(size)), self.lib)
        buf = np.empty(size.value, dtype=np.uint8)
        abi.check(self.lib.sphgpu_checkpoint_save(self.h, _p(buf), size.value), self.lib)
        return buf.tobytes()

    def restore(self, image):
        """SPHHydroBase::restoreState from a checkpoint image of a problem
        with the same configuration and node count."""
        buf = np.frombuffer(image, dtype=np.uint8)
        abi.check(self.lib.sphgpu_checkpoint_load(self.h, _p(buf), buf.size), self.lib)
        self.sync_time()

    def dumpState(self, path, nodeListName="nodes"):
        """The reference's restart file (RestartRegistrar::dumpState through
        FlatFileIO, ascii) of this problem at `path`."""
        abi.check(self.lib.sphgpu_restart_dump(self.h, os.fsencode(str(path)), nodeListName.encode()), self.lib)

    def restoreState(self, path):
        """Restore a restart file in the reference's layout (written by
        dumpState or by the reference itself) and continue from it."""
        abi.check(self.lib.sphgpu_restart_restore(self.h, os.fsencode(str(path))), self.lib)
        self.sync_time()

    def kernel_launches(self):
        v = ctypes.c_int64()
        abi.check(self.lib.sphgpu_kernel_launches(self.h, ctypes.byref(v)), self.lib)
        return v.value

    def sync_time(self):
        t = ctypes.c_double()
        dt = ctypes.c_double()
        abi.check(self.lib.sphgpu_time(self.h, ctypes.byref(t), ctypes.byref(dt)), self.lib)
        self.time = t.value
        return t.value, dt.value

    def set_schedule(self, stage, schedule):
        abi.check(self.lib.sphgpu_set_schedule(self.h, stage.encode(), int(schedule)), self.lib)

    def schedule(self, stage):
        v = ctypes.c_int32()
        abi.check(self.lib.sphgpu_get_schedule(self.h, stage.encode(), ctypes.byref(v)), self.lib)
        return v.value

    def autotune(self):
        """Time every kernel schedule on this problem and keep the fastest."""
        out = np.zeros(8)
        abi.check(self.lib.sphgpu_autotune(self.h, _p(out)), self.lib)
        return _tune_report(out)

    def synchronize(self):
        abi.check(self.lib.sphgpu_synchronize(self.h), self.lib)

    def stream(self):
        s = ctypes.c_void_p()
        abi.check(self.lib.sphgpu_get_stream(self.h, ctypes.byref(s)), self.lib)
        return s.value


class CheapSynchronousRK2Integrator:
    """Drives SPHHydro.step like the reference integrator (one package)."""

    def __init__(self, hydro, dtMin=None, dtMax=None):
        self.hydro = hydro

    def step(self, maxTime=None):
        return self.hydro.step(1)

    def advance(self, nsteps):
        return self.hydro.step(nsteps)


class SPHBatch:
    """Many independent problems advanced together: every stage of every call
    is one kernel launch over all members (no counterpart in the reference,
    whose problems run one at a time).  Members keep their own state; each
    member's results equal those of running it alone."""

    def __init__(self, members):
        self.lib = abi.load_library()
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        h = ctypes.c_void_p()
        abi.check(self.lib.sphgpu_batch_create(arr, len(self.members), ctypes.byref(h)), self.lib)
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.sphgpu_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build_neighbors(self):
        abi.check(self.lib.sphgpu_batch_build_neighbors(self.h), self.lib)

    def evaluateDerivatives(self):
        abi.check(self.lib.sphgpu_batch_evaluate_derivatives(self.h), self.lib)

    def step(self, nsteps=1):
        abi.check(self.lib.sphgpu_batch_step_rk2(self.h, int(nsteps)), self.lib)
        for m in self.members:
            m.sync_time()

    def num_pairs(self):
        v = ctypes.c_int64()
        abi.check(self.lib.sphgpu_batch_pairs(self.h, ctypes.byref(v)), self.lib)
        return v.value

    def pairs_evaluated(self):
        v = ctypes.c_int64()
        abi.check(self.lib.sphgpu_batch_pairs_evaluated(self.h, ctypes.byref(v)), self.lib)
        return v.value

    def kernel_launches(self):
        v = ctypes.c_int64()
        abi.check(self.lib.sphgpu_batch_kernel_launches(self.h, ctypes.byref(v)), self.lib)
        return v.value

    def set_schedule(self, stage, schedule):
        abi.check(self.lib.sphgpu_batch_set_schedule(self.h, stage.encode(), int(schedule)), self.lib)

    def autotune(self):
        out = np.zeros(8)
        abi.check(self.lib.sphgpu_batch_autotune(self.h, _p(out)), self.lib)
        return _tune_report(out)

    def stream(self):
        v = ctypes.c_void_p()
        abi.check(self.lib.sphgpu_batch_get_stream(self.h, ctypes.byref(v)), self.lib)
        return v.value
