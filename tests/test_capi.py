"""The C-ABI libraries load, export every declared symbol, and the host-side table builder
reproduces the reference's halo fill (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden
from licom4py_gpu_b200 import _native, duogrid_gen
from licom4py_gpu_b200.duogrid import make_consts


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^(?:const\s+)?(?:unsigned\s+|long\s+)*\w+\s*\*?\s*((?:bt|ldg)_\w+)\s*\(", text, re.M)))


def test_libbt_exports_every_declared_symbol():
    lib = _native.lib()
    names = _declared("licom_bt.h")
    assert "bt_round" in names and "bt_plan_create" in names
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_native.EXPORTS)
    assert lib.bt_version() >= 1


def test_libduogrid_exports_every_declared_symbol():
    lib = duogrid_gen._load()
    for name in _declared("licom_duogrid.h"):
        assert hasattr(lib, name), name


def test_plan_create_rejects_bad_descriptor():
    lib = _native.lib()
    desc = _native.GridDesc(2, _native.BT_F64)  # n too small, NULL pointers
    h = ctypes.c_void_p()
    rc = lib.bt_plan_create(ctypes.byref(desc), ctypes.byref(h))
    assert rc == _native.BT_EINVAL
    assert b"n must be" in lib.bt_last_error()
    with pytest.raises(ValueError):
        _native.check(rc)


def _fake_desc(misaligned):
    """A descriptor with non-NULL placeholder pointers (never dereferenced: the
    argument checks come first); ``misaligned`` names one pointer set 8 bytes
    off a 16-byte boundary."""
    desc = _native.GridDesc(48, _native.BT_F64)
    for k, (name, _) in enumerate(_native.GridDesc._fields_[2:]):
        setattr(desc, name, 0x10000 + 0x1000 * k + (8 if name == misaligned else 0))
    return desc


@pytest.mark.parametrize("name", ["a_c2l", "a_l2c", "a_gct"])
def test_matrix_arrays_must_be_16_byte_aligned(name):
    lib = _native.lib()
    h = ctypes.c_void_p()
    rc = lib.bt_plan_create(ctypes.byref(_fake_desc(name)), ctypes.byref(h))
    assert rc == _native.BT_EINVAL and not h.value
    assert b"16-byte aligned" in lib.bt_last_error()
    sin, sout = _native.StateIn(), _native.StateOut()
    rc = lib.bt_round_noalloc(ctypes.byref(_fake_desc(name)), ctypes.byref(sin), ctypes.byref(sout), 1, 10.0, 2, None)
    assert rc == _native.BT_EINVAL
    assert b"16-byte aligned" in lib.bt_last_error()


def halo_tables(n, grid):
    c = make_consts(grid, 5000.0)
    m = n + 6
    nh = 12 * n + 36
    src = np.zeros((6, nh, 2), dtype=np.int32)
    w = np.zeros((6, nh, 2), dtype=np.float64)
    route = np.zeros(24, dtype=np.int32)
    coef = np.ascontiguousarray(c[5])
    li = np.ascontiguousarray(c[6])
    lj = np.ascontiguousarray(c[7])
    rc = _native.lib().bt_halo_table_host(n, coef.ctypes.data, li.ctypes.data, lj.ctypes.data,
                                          src.ctypes.data, w.ctypes.data, route.ctypes.data)
    _native.check(rc)
    return src, w, route, c


def halo_cells(m):
    """(i, j) of halo ids 0..nh-1 (order of include/licom_bt.h)."""
    n = m - 6
    cells = [(i, j) for i in range(3) for j in range(m)]
    cells += [(i, j) for i in range(m - 3, m) for j in range(m)]
    cells += [(i, j) for i in range(3, m - 3) for j in range(3)]
    cells += [(i, j) for i in range(3, m - 3) for j in range(m - 3, m)]
    assert len(cells) == 12 * n + 36
    return cells


@pytest.mark.parametrize("n", [8, 12])
def test_host_halo_table_reproduces_ext_scalar_and_ext_vector(n, grids):
    z = load_golden("halo.npz")
    src, w, route, c = halo_tables(n, grids(n))
    m = n + 6
    s = z[f"c{n}_s"]
    u, v = z[f"c{n}_u"], z[f"c{n}_v"]
    out = s.copy()
    uo, vo = u.copy(), v.copy()
    flat, fu, fv = s.ravel(), u.ravel(), v.ravel()
    c2l = c[8].reshape(-1, 2, 2)
    l2c = c[9]
    for f in range(6):
        for hid, (i, j) in enumerate(halo_cells(m)):
            s0, s1 = src[f, hid]
            w0, w1 = w[f, hid]
            out[f, i, j] = w0 * flat[s0] + w1 * flat[s1]
            ull0 = c2l[s0, 0, 0] * fu[s0] + c2l[s0, 0, 1] * fv[s0]
            vll0 = c2l[s0, 1, 0] * fu[s0] + c2l[s0, 1, 1] * fv[s0]
            ull1 = c2l[s1, 0, 0] * fu[s1] + c2l[s1, 0, 1] * fv[s1]
            vll1 = c2l[s1, 1, 0] * fu[s1] + c2l[s1, 1, 1] * fv[s1]
            ull = w0 * ull0 + w1 * ull1
            vll = w0 * vll0 + w1 * vll1
            L = l2c[f, i, j]
            uo[f, i, j] = L[0, 0] * ull + L[0, 1] * vll
            vo[f, i, j] = L[1, 0] * ull + L[1, 1] * vll
    np.testing.assert_array_equal(out, z[f"c{n}_ext_scalar"])
    np.testing.assert_array_equal(uo, z[f"c{n}_ext_u"])
    np.testing.assert_array_equal(vo, z[f"c{n}_ext_v"])
    # routing entries nb | side << 4 | rev << 6 against Communication._routing
    r = z[f"c{n}_routing"]
    for t in range(6):
        for d in range(4):
            e = int(route[t * 4 + d])
            assert (e & 15, (e >> 4) & 3, (e >> 6) & 1) == tuple(int(x) for x in r[t, d])


def test_host_halo_table_rejects_corrupt_locations(grids):
    n = 8
    c = make_consts(grids(n), 5000.0)
    li = np.ascontiguousarray(c[6]).copy()
    li[0, 5, 0] = 999
    nh = 12 * n + 36
    src = np.zeros((6, nh, 2), np.int32)
    w = np.zeros((6, nh, 2))
    route = np.zeros(24, np.int32)
    coef = np.ascontiguousarray(c[5])
    lj = np.ascontiguousarray(c[7])
    rc = _native.lib().bt_halo_table_host(n, coef.ctypes.data, li.ctypes.data, lj.ctypes.data,
                                          src.ctypes.data, w.ctypes.data, route.ctypes.data)
    assert rc == _native.BT_EINVAL
    assert b"out of range" in _native.lib().bt_last_error()
