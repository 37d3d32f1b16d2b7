"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and call the CUDA path
through the C-ABI; everything else runs on the CPU (oracle, host logic,
library loading)."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the CUDA path through the C-ABI")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("llnl-spheral_b200")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_lib(pkg):
    """The CUDA library; a GPU test must not run without it."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    from importlib import import_module
    build = import_module("llnl-spheral_b200.build")
    build.build()
    return pkg.abi.load_library()


def normwise(a, b):
    """||a - b||_inf / ||b||_inf (plain ||a - b||_inf when b == 0)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b)) if b.size else 0.0
    d = np.max(np.abs(a - b)) if b.size else 0.0
    return d / s if s > 0 else d
