"""TEST INFRASTRUCTURE: ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs use this module, and only as the checker or the timed CPU reference.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        L.orc_create.restype = P
        L.orc_create.argtypes = [P, ctypes.c_int] + [P] * 6
        L.orc_destroy.argtypes = [P]
        L.orc_last_error.restype = ctypes.c_char_p
        for n in ("orc_build_neighbors", "orc_num_ghosts", "orc_initialize", "orc_evaluate_derivatives",
                  "orc_finalize"):
            getattr(L, n).argtypes = [P]
        L.orc_num_entries.argtypes = [P]
        L.orc_num_entries.restype = ctypes.c_int64
        L.orc_num_pairs.argtypes = [P]
        L.orc_num_pairs.restype = ctypes.c_int64
        L.orc_get_connectivity.argtypes = [P, P, P, P]
        L.orc_get_ghost_positions.argtypes = [P, P]
        L.orc_dt.argtypes = [P]
        L.orc_dt.restype = ctypes.c_double
        L.orc_step_rk2.argtypes = [P, ctypes.c_int, P, P]
        L.orc_iterate_ideal_h.argtypes = [P, ctypes.c_int, ctypes.c_double, P]
        L.orc_get_field.argtypes = [P, ctypes.c_char_p, P]
        L.orc_get_pair_accelerations.argtypes = [P, P]
        L.orc_conservation.argtypes = [P, P]
        L.orc_table_create.restype = P
        L.orc_table_create.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_table_destroy.argtypes = [P]
        L.orc_table_coeffs.argtypes = [P, P]
        L.orc_table_eval.argtypes = [P, ctypes.c_int, P, ctypes.c_double, P, P, P]
        L.orc_base_kernel.restype = ctypes.c_double
        L.orc_base_kernel.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_geometry.argtypes = [ctypes.c_int, P, P, P]
        L.orc_map_positions.argtypes = [ctypes.c_int, P, P, P, ctypes.c_int, ctypes.c_int, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


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


class OracleProblem:
    """One FluidNodeList in a periodic box, evolved by the CPU oracle."""

    def __init__(self, cfg, nodes):
        self.L = lib()
        self.n = nodes.n
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in
                      (nodes.pos, nodes.vel, nodes.mass, nodes.rho, nodes.eps, nodes.H)]
        self.h = self.L.orc_create(ctypes.byref(cfg), self.n, *[_p(a) for a in self._keep])

    def __del__(self):
        try:
            self.L.orc_destroy(self.h)
        except Exception:
            pass

    def build_neighbors(self):
        self.L.orc_build_neighbors(self.h)

    def num_ghosts(self):
        return self.L.orc_num_ghosts(self.h)

    def num_pairs(self):
        return self.L.orc_num_pairs(self.h)

    def connectivity(self):
        e = self.L.orc_num_entries(self.h)
        off = np.zeros(self.n + 1, dtype=np.int64)
        nb = np.zeros(max(e, 1), dtype=np.int32)
        root = np.zeros(max(self.num_ghosts(), 1), dtype=np.int32)
        self.L.orc_get_connectivity(self.h, _p(off), _p(nb), _p(root))
        return off, nb[:e], root[:self.num_ghosts()]

    def pair_accelerations(self):
        """The reference's pair-wise accelerations, (E, 3) in row order."""
        e = self.L.orc_num_entries(self.h)
        out = np.zeros((max(e, 1), 3))
        self.L.orc_get_pair_accelerations(self.h, _p(out))
        return out[:e]

    def ghost_positions(self):
        g = np.zeros((max(self.num_ghosts(), 1), 3))
        self.L.orc_get_ghost_positions(self.h, _p(g))
        return g[:self.num_ghosts()]

    def initialize(self):
        self.L.orc_initialize(self.h)

    def evaluate_derivatives(self):
        self.L.orc_evaluate_derivatives(self.h)

    def finalize(self):
        self.L.orc_finalize(self.h)

    def dt(self):
        return self.L.orc_dt(self.h)

    def step(self, nsteps=1):
        t = ctypes.c_double()
        dt = ctypes.c_double()
        rc = self.L.orc_step_rk2(self.h, nsteps, ctypes.byref(t), ctypes.byref(dt))
        if rc != 0:
            raise RuntimeError("oracle step failed: %s" % self.L.orc_last_error().decode())
        return t.value, dt.value

    def iterate_ideal_h(self, max_iterations=50, tolerance=1.0e-4):
        dh = ctypes.c_double()
        itr = self.L.orc_iterate_ideal_h(self.h, int(max_iterations), float(tolerance), ctypes.byref(dh))
        return itr, dh.value

    def field(self, key):
        c = FIELD_COMPONENTS[key]
        out = np.zeros(self.n * c)
        rc = self.L.orc_get_field(self.h, key.encode(), _p(out))
        if rc != 0:
            raise KeyError(key)
        return out.reshape(self.n, c) if c > 1 else out

    def conservation(self):
        out = np.zeros(8)
        self.L.orc_conservation(self.h, _p(out))
        return out


class OracleTable:
    def __init__(self, kernel_type, num_points):
        self.L = lib()
        self.n = num_points
        self.h = self.L.orc_table_create(kernel_type, num_points)

    def __del__(self):
        try:
            self.L.orc_table_destroy(self.h)
        except Exception:
            pass

    def coeffs(self):
        out = np.zeros(11 * self.n)
        self.L.orc_table_coeffs(self.h, _p(out))
        return out.reshape(11, self.n)

    def eval(self, eta, Hdet=1.0):
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        W = np.zeros_like(eta)
        gW = np.zeros_like(eta)
        self.L.orc_table_eval(self.h, eta.size, _p(eta), Hdet, _p(W), _p(gW), None)
        return W, gW

    def nperh(self, wsum):
        wsum = np.ascontiguousarray(wsum, dtype=np.float64)
        out = np.zeros_like(wsum)
        self.L.orc_table_eval(self.h, wsum.size, _p(wsum), 1.0, None, None, _p(out))
        return out
