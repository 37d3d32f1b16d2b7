"""Pin the CPU oracle to the reference itself.

tests/golden/reference_tables.npz holds outputs of the reference's own
TableKernel, BSpline/Wendland C4 kernels, Dim<3> geometry and
mapPositionThroughPlanes, compiled unmodified from the reference tree
(oracle/build_ref.py, tests/golden/make_golden.py).  The oracle must
reproduce them bit for bit.
"""
import ctypes
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_tables.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("tag,ktype", [("bspline", 0), ("wendlandc4", 1)])
def test_table_kernel_bitexact(oracle_mod, golden, tag, ktype):
    T = oracle_mod.OracleTable(ktype, 1000)
    W, gW = T.eval(golden[tag + "_eta"])
    assert np.array_equal(W, golden[tag + "_W"])
    assert np.array_equal(gW, golden[tag + "_gW"])
    co = T.coeffs()
    assert np.array_equal(co[9], golden[tag + "_nperh"])
    assert np.array_equal(co[10], golden[tag + "_wsum"])
    assert np.array_equal(T.nperh(golden[tag + "_wsum_query"]), golden[tag + "_nperh_query"])


@pytest.mark.parametrize("tag,ktype", [("bspline", 0), ("wendlandc4", 1)])
def test_analytic_kernels_bitexact(oracle_mod, golden, tag, ktype):
    L = oracle_mod.lib()
    eta = golden[tag + "_eta"]
    an = golden[tag + "_analytic"].reshape(-1, 2)
    ours = np.array([[L.orc_base_kernel(ktype, 0, e), L.orc_base_kernel(ktype, 1, e)] for e in eta[:800]])
    assert np.array_equal(ours, an[:800])


def test_geometry_bitexact(oracle_mod, golden):
    L = oracle_mod.lib()
    H = np.ascontiguousarray(golden["geom_H"])
    r = np.ascontiguousarray(golden["geom_r"])
    n = r.size // 3
    out = np.zeros(16 * n)
    L.orc_geometry(n, _p(H), _p(r), _p(out))
    assert np.array_equal(out, golden["geom_out"])


def test_periodic_plane_mapping_bitexact(oracle_mod, golden):
    L = oracle_mod.lib()
    pin = np.ascontiguousarray(golden["map_in"])
    m = pin.size // 3
    lo = np.array([0.0, 0.0, 0.0])
    hi = np.array([1.0, 0.125, 0.125])
    res = []
    for axis in range(3):
        for which in range(2):
            o = np.zeros(3 * m)
            L.orc_map_positions(m, _p(pin), _p(lo), _p(hi), axis, which, _p(o))
            res.append(o)
    assert np.array_equal(np.concatenate(res), golden["map_out"])
