"""sphgpu_conservation_noalloc against sphgpu_conservation.

The no-allocation entry point sums over caller-owned device arrays with its
scratch in a fixed device array of the library.  It must agree with the
handle-based sphgpu_conservation within 1e-12 (relative to the sum of
magnitudes of each component: the two use different summation orders), on
two calls in a row, and reject node counts beyond its scratch limit.
This file is collected last so that it also runs after every other GPU test
has used the device.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_NODES = 8192 * 2048


def _device_state(torch, g):
    m = torch.from_numpy(np.ascontiguousarray(g.field("mass"))).cuda()
    v = torch.from_numpy(np.ascontiguousarray(g.field("velocity")).reshape(-1)).cuda()
    e = torch.from_numpy(np.ascontiguousarray(g.field("specific thermal energy"))).cuda()
    torch.cuda.synchronize()
    return m, v, e


def _noalloc(lib, m, v, e, n, stream=None):
    out = np.full(8, np.nan)
    rc = lib.sphgpu_conservation_noalloc(ctypes.c_void_p(m.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                         ctypes.c_void_p(e.data_ptr()), n,
                                         None if stream is None else ctypes.c_void_p(stream.cuda_stream),
                                         out.ctypes.data_as(ctypes.c_void_p))
    return rc, out


def _scales(g):
    m = g.field("mass")
    v = g.field("velocity")
    e = g.field("specific thermal energy")
    ke = 0.5 * m * (v * v).sum(axis=1)
    s = [m.sum(), *(m[:, None] * np.abs(v)).sum(axis=0), ke.sum(), np.abs(m * e).sum()]
    return np.array(s + [s[4] + s[5], 1.0])


@pytest.mark.parametrize("shape", [(24, 24, 12), (64, 64, 64)])
def test_noalloc_matches_handle_conservation(gpu_lib, pkg, shape):
    import torch
    gen, abi = pkg.generators, pkg.abi
    nx, ny, nz = shape
    ns = gen.kelvin_helmholtz(nx=nx, ny=ny, nz=nz, box=((0, 0, 0), (1.0, 1.0, nz / nx)))
    cfg = gen.kh_config(abi, xmax=(1.0, 1.0, nz / nx))
    g = pkg.SPHHydro(cfg, ns)
    if ns.n < 50000:
        g.step(2)
    ref = g.conservation()
    scale = _scales(g)
    m, v, e = _device_state(torch, g)
    rc1, out1 = _noalloc(gpu_lib, m, v, e, ns.n)
    rc2, out2 = _noalloc(gpu_lib, m, v, e, ns.n)
    assert rc1 == 0 and rc2 == 0, gpu_lib.sphgpu_last_error()
    for out in (out1, out2):
        assert np.all(np.abs(out - ref) <= 1e-12 * scale), (out, ref)
    assert np.array_equal(out1, out2)


def test_noalloc_on_a_caller_stream(gpu_lib, pkg):
    """A serving loop passes its own stream: the sums are the same bits as on
    the default stream, call after call."""
    import torch
    gen, abi = pkg.generators, pkg.abi
    ns = gen.kelvin_helmholtz(nx=32, ny=32, nz=16, box=((0, 0, 0), (1.0, 1.0, 0.5)))
    g = pkg.SPHHydro(gen.kh_config(abi, xmax=(1.0, 1.0, 0.5)), ns)
    m, v, e = _device_state(torch, g)
    rc0, base = _noalloc(gpu_lib, m, v, e, ns.n)
    assert rc0 == 0, gpu_lib.sphgpu_last_error()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    for _ in range(2):
        rc, out = _noalloc(gpu_lib, m, v, e, ns.n, stream=s)
        assert rc == 0, gpu_lib.sphgpu_last_error()
        assert np.array_equal(out, base)


def test_noalloc_rejects_sizes_beyond_scratch(gpu_lib):
    import torch
    m = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc, out = _noalloc(gpu_lib, m, m, m, MAX_NODES + 1)
    assert rc == -3
    assert b"16,777,216" in gpu_lib.sphgpu_last_error()
    assert np.all(np.isnan(out))
    rc, out = _noalloc(gpu_lib, m, m, m, -1)
    assert rc == -1


def test_noalloc_empty(gpu_lib):
    import torch
    m = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc, out = _noalloc(gpu_lib, m, m, m, 0)
    assert rc == 0
    assert np.all(out == 0.0)
