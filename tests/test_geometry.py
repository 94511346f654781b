"""Invariants of the generated duogrid geometry (the reference ships no grid file to compare with)."""
import math

import numpy as np
import pytest

from licom4py_gpu_b200 import duogrid_gen
from licom4py_gpu_b200.duogrid import Duogrid, make_consts

R = 6.3712e6
H = 3


@pytest.mark.parametrize("n", [8, 24, 48])
def test_area_sums_to_sphere(n, grids):
    g = duogrid_gen.generate(n, fields=["a_da"])
    total = g["a_da"][:, H:-H, H:-H].sum()
    assert abs(total / (4 * math.pi * R * R) - 1.0) < 1e-11


@pytest.mark.parametrize("n", [8, 48])
def test_c2l_l2c_inverse(n, grids):
    g = grids(n)
    prod = np.einsum("...ab,...bc->...ac", g["a_c2l"], g["a_l2c"])
    assert np.abs(prod - np.eye(2)).max() < 1e-13


@pytest.mark.parametrize("n", [8, 48])
def test_k2e_tables(n, grids):
    g = grids(n)
    m = n + 6
    li, lj, coef = g["k2e_loc_i"], g["k2e_loc_j"], g["k2e_coef"]
    np.testing.assert_array_equal(li, lj)  # both are k2e_loc - isd (isd = jsd = -2)
    bands = [li[:, H:m - H, :H], li[:, H:m - H, m - H:], lj[:, :H, H:m - H], lj[:, m - H:, H:m - H]]
    for b in bands:
        assert b.min() >= H and b.max() <= m - H - 2
    cb = [coef[:, H:m - H, :H], coef[:, H:m - H, m - H:], coef[:, :H, H:m - H], coef[:, m - H:, H:m - H]]
    for c in cb:
        np.testing.assert_allclose(c.sum(-1), 1.0, atol=1e-14)
    # identical on all six faces (the equal-edge grid is face independent)
    for f in range(1, 6):
        np.testing.assert_array_equal(li[f], li[0])
        np.testing.assert_array_equal(coef[f], coef[0])


def test_metric_symmetry(grids):
    g = grids(24)
    rdx, rdy = g["rdx"], g["rdy"]
    np.testing.assert_array_equal(rdx[0], rdy[0].T)      # dx(i,j) = dy(j,i)
    np.testing.assert_array_equal(rdx[0], rdx[3])        # face independent
    assert np.all(g["a_sina"][:, H:-H, H:-H] > 0.8)


def test_coriolis_and_points(grids):
    g = grids(24)
    lat = g["a_pt"][..., 1]
    np.testing.assert_allclose(g["a_f"], 2 * 7.292e-5 * np.sin(lat), rtol=0, atol=1e-18)
    assert np.all(np.abs(lat) <= math.pi / 2 + 1e-12)


def test_generator_rejects_bad_resolution():
    with pytest.raises(duogrid_gen.DuogridError):
        duogrid_gen.generate(3)


def test_npz_roundtrip_and_configure(tmp_path):
    path = duogrid_gen.DuogridFieldGenerator(8, out_dir=str(tmp_path)).run()
    assert path.endswith("duogrid_C8.npz")
    with np.load(path) as z:
        assert set(z.files) == set(duogrid_gen.ESSENTIAL_FIELDS)
    Dg = Duogrid.configure(8, npz_path=path, depth=5000.0)
    assert Dg.inner.sum() == 6 * 64 and Dg.dzph_x[0, 0, 0] == 5000.0
    with pytest.raises(FileNotFoundError):
        Duogrid.configure(8, npz_path=str(tmp_path / "missing.npz"))


def test_make_consts_order(grids):
    c = make_consts(grids(8), 5600.0)
    assert len(c) == 17
    assert c[6].dtype == np.int32 and c[7].dtype == np.int32
    assert c[0][0, 0, 0] == 5600.0


def _halo_fill_error(n, grids):
    """Max error of the duogrid halo fill (the host gather table: two interior sources, two
    weights per halo cell) of a smooth analytic field against the field at the halo points, over
    the halo cells beside the face edges.  The 3 x 3 corner blocks are excluded: the reference
    fills them by copying the adjacent band cell, not by interpolation."""
    from test_capi import halo_cells, halo_tables
    g = grids(n)
    src, w, _, _ = halo_tables(n, g)
    lon, lat = g["a_pt"][..., 0], g["a_pt"][..., 1]
    field = np.cos(lat) * np.cos(lon - 0.3) + 0.5 * np.sin(lat) ** 2  # smooth on the sphere
    flat = field.reshape(-1)
    m = n + 6
    err = 0.0
    for f in range(6):
        for k, (i, j) in enumerate(halo_cells(m)):
            if (i < H or i >= m - H) and (j < H or j >= m - H):
                continue
            a, b = src[f, k]
            got = w[f, k, 0] * flat[a] + w[f, k, 1] * flat[b]
            err = max(err, abs(got - field[f, i, j]))
    return err


def test_halo_fill_of_a_smooth_field_is_second_order(grids):
    """The halo fill (update_domain + the linear cube_rmp remap) interpolates linearly: its error on a
    smooth field of unit size is small and falls about 4x when the resolution doubles."""
    e24, e48 = _halo_fill_error(24, grids), _halo_fill_error(48, grids)
    assert e48 < 1e-3
    assert e24 / e48 > 3.5, (e24, e48)
