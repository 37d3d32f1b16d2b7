"""ctypes mirror of include/sphgpu.h and loader of the native library.

The native library ``_build/libsphgpu.so`` (CUDA sm_100a kernels + the C-ABI)
is built in-tree by ``build.py``.  Importing the product path fails loudly when
the library is missing: there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsphgpu.so")

# status codes
OK = 0
ERR_ARG, ERR_CUDA, ERR_CAPACITY, ERR_STATE, ERR_UNSUPPORTED, ERR_NUMERIC, ERR_NOMEM, ERR_ADMISSION = \
    -1, -2, -3, -4, -5, -6, -7, -8

HYDRO_SPH, HYDRO_CRKSPH = 0, 1
KERNEL_BSPLINE, KERNEL_WENDLANDC4 = 0, 1
DENSITY_RIGOROUS_SUM, DENSITY_INTEGRATE = 0, 1
H_IDEAL, H_INTEGRATE = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
CRK_SUMVOLUME, CRK_MASSOVERDENSITY = 0, 1
Q_MONAGHAN_GINGOLD, Q_CRKSPH_MONAGHAN_GINGOLD = 0, 1


class SphConfig(ctypes.Structure):
    """Layout-identical to ``sphgpu_config``."""
    _fields_ = [
        ("hydro", ctypes.c_int32),
        ("kernel", ctypes.c_int32),
        ("num_points", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("nPerh", ctypes.c_double),
        ("Cl", ctypes.c_double),
        ("Cq", ctypes.c_double),
        ("epsilon2", ctypes.c_double),
        ("linearInExpansion", ctypes.c_int32),
        ("quadraticInExpansion", ctypes.c_int32),
        ("cfl", ctypes.c_double),
        ("epsTensile", ctypes.c_double),
        ("nTensile", ctypes.c_double),
        ("hmin", ctypes.c_double),
        ("hmax", ctypes.c_double),
        ("hminratio", ctypes.c_double),
        ("rhoMin", ctypes.c_double),
        ("rhoMax", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("compatibleEnergyEvolution", ctypes.c_int32),
        ("gradhCorrection", ctypes.c_int32),
        ("XSPH", ctypes.c_int32),
        ("correctVelocityGradient", ctypes.c_int32),
        ("densityUpdate", ctypes.c_int32),
        ("HUpdate", ctypes.c_int32),
        ("useVelocityMagnitudeForDt", ctypes.c_int32),
        ("crkVolumeType", ctypes.c_int32),
        ("xmin", ctypes.c_double * 3),
        ("xmax", ctypes.c_double * 3),
        ("periodic", ctypes.c_int32 * 3),
        ("max_neighbors", ctypes.c_int32),
        ("dtMin", ctypes.c_double),
        ("dtMax", ctypes.c_double),
        ("dtGrowth", ctypes.c_double),
        ("lastDt", ctypes.c_double),
        ("qType", ctypes.c_int32),
        ("balsaraShearCorrection", ctypes.c_int32),
        ("etaCritFrac", ctypes.c_double),
        ("etaFoldFrac", ctypes.c_double),
    ]

    def copy(self):
        c = SphConfig()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(SphConfig))
        return c


def make_config(**kw):
    """A config with the reference's C++/factory defaults; keywords override.

    Defaults follow SPHHydroBase's Python factory (src/SPH/SPHHydros.py:14-31)
    with the hot-path switches pinned explicitly, MonaghanGingoldViscosity
    (Cl = Cq = 1, epsilon2 = 1e-2 from ArtificialViscosity.cc:42-90) and the
    FluidNodeList factory limits (src/NodeList/FluidNodeLists.py:11-35).
    """
    c = SphConfig()
    c.hydro = HYDRO_SPH
    c.kernel = KERNEL_BSPLINE
    c.num_points = 1000
    c.precision = PRECISION_FP64
    c.nPerh = 1.51
    c.Cl, c.Cq, c.epsilon2 = 1.0, 1.0, 1.0e-2
    c.linearInExpansion = 0
    c.quadraticInExpansion = 0
    c.cfl = 0.25
    c.epsTensile, c.nTensile = 0.0, 4.0
    c.hmin, c.hmax, c.hminratio = 1.0e-20, 1.0e20, 0.1
    c.rhoMin, c.rhoMax = 1.0e-10, 1.0e10
    c.gamma = 5.0 / 3.0
    c.compatibleEnergyEvolution = 1
    c.gradhCorrection = 0
    c.XSPH = 0
    c.correctVelocityGradient = 1
    c.densityUpdate = DENSITY_RIGOROUS_SUM
    c.HUpdate = H_IDEAL
    c.useVelocityMagnitudeForDt = 0
    c.crkVolumeType = CRK_SUMVOLUME
    for a in range(3):
        c.xmin[a], c.xmax[a], c.periodic[a] = 0.0, 1.0, 1
    c.max_neighbors = 0
    c.dtMin, c.dtMax, c.dtGrowth, c.lastDt = 0.0, 0.1, 2.0, 1.0e-5
    # CRKSPHMonaghanGingoldViscosity constructor defaults
    # (src/PBGWraps/ArtificialViscosity/ArtificialViscosityModule.py:209-214)
    c.qType = Q_MONAGHAN_GINGOLD
    c.etaCritFrac, c.etaFoldFrac = 1.0, 0.2
    for k, v in kw.items():
        if k in ("xmin", "xmax", "periodic"):
            for a in range(3):
                getattr(c, k)[a] = v[a]
        else:
            if not hasattr(c, k):
                raise AttributeError("unknown config field %s" % k)
            setattr(c, k, v)
    return c


_lib = None


def load_library(path=None):
    """Load libsphgpu.so (CUDA build).  Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("libsphgpu.so not built (%s); run build.py / __graft_entry__.build()" % p)
    lib = ctypes.CDLL(p)
    P = ctypes.c_void_p
    D = ctypes.POINTER(ctypes.c_double)
    I64 = ctypes.c_int64
    lib.sphgpu_last_error.restype = ctypes.c_char_p
    lib.sphgpu_create.argtypes = [ctypes.POINTER(SphConfig), I64, ctypes.POINTER(P)]
    lib.sphgpu_destroy.argtypes = [P]
    lib.sphgpu_destroy.restype = None
    for name in ("sphgpu_set_state", "sphgpu_set_state_device", "sphgpu_get_state"):
        getattr(lib, name).argtypes = [P] + [P] * 6
    lib.sphgpu_get_field.argtypes = [P, ctypes.c_char_p, P, I64]
    lib.sphgpu_field_components.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32)]
    lib.sphgpu_build_neighbors.argtypes = [P]
    lib.sphgpu_connectivity_size.argtypes = [P, ctypes.POINTER(I64), ctypes.POINTER(I64)]
    lib.sphgpu_get_connectivity.argtypes = [P, P, P, P]
    lib.sphgpu_get_ghost_positions.argtypes = [P, P]
    lib.sphgpu_get_pair_accelerations.argtypes = [P, P, I64]
    for name in ("sphgpu_initialize", "sphgpu_evaluate_derivatives", "sphgpu_finalize_derivatives",
                 "sphgpu_finalize"):
        getattr(lib, name).argtypes = [P, ctypes.c_double, ctypes.c_double]
    lib.sphgpu_dt.argtypes = [P, D]
    lib.sphgpu_step_rk2.argtypes = [P, D, I64, D]
    lib.sphgpu_step_rk2_host.argtypes = [P] + [P] * 12 + [D, D]
    lib.sphgpu_conservation.argtypes = [P, P]
    lib.sphgpu_iterate_ideal_h.argtypes = [P, ctypes.c_int32, ctypes.c_double, ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_double)]
    lib.sphgpu_checkpoint_size.argtypes = [P, ctypes.POINTER(I64)]
    lib.sphgpu_checkpoint_save.argtypes = [P, P, I64]
    lib.sphgpu_checkpoint_load.argtypes = [P, P, I64]
    lib.sphgpu_restart_dump.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p]
    lib.sphgpu_restart_restore.argtypes = [P, ctypes.c_char_p]
    lib.sphgpu_restart_labels.argtypes = [ctypes.POINTER(SphConfig), ctypes.c_char_p, I64]
    lib.sphgpu_set_field.argtypes = [P, ctypes.c_char_p, P, I64]
    lib.sphgpu_set_dt_bounds.argtypes = [P, ctypes.c_double, ctypes.c_double]
    lib.sphgpu_num_pairs.argtypes = [P, ctypes.POINTER(I64)]
    lib.sphgpu_pairs_evaluated.argtypes = [P, ctypes.POINTER(I64)]
    lib.sphgpu_kernel_launches.argtypes = [P, ctypes.POINTER(I64)]
    lib.sphgpu_time.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.sphgpu_batch_create.argtypes = [P, ctypes.c_int32, ctypes.POINTER(P)]
    lib.sphgpu_batch_destroy.argtypes = [P]
    lib.sphgpu_batch_destroy.restype = None
    lib.sphgpu_batch_size.argtypes = [P, ctypes.POINTER(ctypes.c_int32)]
    lib.sphgpu_batch_build_neighbors.argtypes = [P]
    lib.sphgpu_batch_evaluate_derivatives.argtypes = [P]
    lib.sphgpu_batch_step_rk2.argtypes = [P, I64]
    lib.sphgpu_batch_pairs.argtypes = [P, ctypes.POINTER(I64)]
    lib.sphgpu_batch_pairs_evaluated.argtypes = [P, ctypes.POINTER(I64)]
    lib.sphgpu_batch_kernel_launches.argtypes = [P, ctypes.POINTER(I64)]
    lib.sphgpu_batch_set_schedule.argtypes = [P, ctypes.c_char_p, ctypes.c_int32]
    lib.sphgpu_batch_get_stream.argtypes = [P, ctypes.POINTER(P)]
    lib.sphgpu_autotune.argtypes = [P, P]
    lib.sphgpu_batch_autotune.argtypes = [P, P]
    lib.sphgpu_estimate_footprint.argtypes = [P, I64, P, P, ctypes.POINTER(I64)]
    lib.sphgpu_server_create.argtypes =[ctypes.c_double, ctypes.c_int32, ctypes.POINTER(P)]
    lib.sphgpu_server_destroy.argtypes = [P]
    lib.sphgpu_server_destroy.restype = None
    lib.sphgpu_server_submit.argtypes = [P, P, I64] + [P] * 6 + [I64, ctypes.POINTER(I64)]
    lib.sphgpu_server_tick.argtypes = [P, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    lib.sphgpu_server_finished.argtypes = [P, P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    lib.sphgpu_server_cancel.argtypes = [P, I64]
    lib.sphgpu_server_status.argtypes = [P, I64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(I64),
                                         ctypes.POINTER(I64)]
    lib.sphgpu_server_fetch.argtypes = [P, I64] + [P] * 6 + [ctypes.POINTER(ctypes.c_double)]
    lib.sphgpu_server_stats.argtypes = [P, P]
    lib.sphgpu_conservation_noalloc.argtypes = [P, P, P, I64, P, P]
    lib.sphgpu_set_schedule.argtypes = [P, ctypes.c_char_p, ctypes.c_int32]
    lib.sphgpu_get_schedule.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32)]
    lib.sphgpu_synchronize.argtypes = [P]
    lib.sphgpu_get_stream.argtypes = [P, ctypes.POINTER(P)]
    lib.sphgpu_set_stream.argtypes = [P, P]
    _lib = lib
    return lib


def check(rc, lib=None):
    if rc != OK:
        lib = lib or _lib
        msg = lib.sphgpu_last_error().decode() if lib is not None else ""
        raise RuntimeError("sphgpu error %d: %s" % (rc, msg))
    return rc


def restart_labels(cfg):
    """Unique labels, in order, of the objects a restart file of `cfg` holds
    (sphgpu_restart_labels; host only)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(4096)
    check(lib.sphgpu_restart_labels(ctypes.byref(cfg), buf, len(buf)), lib)
    return buf.value.decode().split()
