"""B200-native SPH/CRKSPH fluid-hydro derivative path (drop-in for Spheral's
SPHHydroBase / CRKSPHHydroBase evaluateDerivatives and the RK2 step).

The package directory holds the CUDA sources (csrc/), the in-tree build
(build.py -> _build/libsphgpu.so), the ctypes mirror of include/sphgpu.h
(abi.py), the host-side hydro interface (hydro.py), the serving loop
(serving.py), the placement of independent problems on the GPUs of a node
(sharding.py) and seeded node generators for the benchmark shapes
(generators.py).

Import with ``importlib.import_module("llnl-spheral_b200")`` (the directory
name carries a hyphen).
"""
from . import abi  # noqa: F401
from . import generators  # noqa: F401
from . import hydro  # noqa: F401
from .hydro import SPHHydro, SPHBatch, CheapSynchronousRK2Integrator  # noqa: F401
from . import serving  # noqa: F401
from . import sharding  # noqa: F401
from . import domains  # noqa: F401
