"""Seeded synthetic initial states and the CFL step."""
import math

import numpy as np

from licom4py_gpu_b200.fields import cfl_dtb, harmonic_series, harmonic_state, w92_case2_state

H = 3


def test_harmonic_state_rms_and_determinism(grids):
    g = grids(24)
    a = harmonic_state(g, 5)
    b = harmonic_state(g, 5)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert abs(math.sqrt(np.mean(a["h0"][:, H:-H, H:-H] ** 2)) - 1.0) < 1e-12
    c = harmonic_state(g, 6)
    assert not np.array_equal(a["h0"], c["h0"])


def test_harmonics_are_orthonormal_enough(grids):
    # integral of Y_lm^2 over the sphere ~ 1 for a single unit coefficient series
    g = grids(48)
    lon, lat = g["a_pt"][..., 0], g["a_pt"][..., 1]
    da = 1.0 / g["rda"]
    f = harmonic_series(lon, lat, seed=0, lmin=1, lmax=1)
    rng = np.random.default_rng(0)
    c = rng.standard_normal(3)
    R2 = 6.3712e6 ** 2
    integral = (f[:, H:-H, H:-H] ** 2 * da[:, H:-H, H:-H]).sum() / R2
    assert abs(integral / (c ** 2).sum() - 1.0) < 1e-3


def test_cfl_dtb_values(grids):
    # about 0.5 * 1.231 R / N / sqrt(g H) for the equal-edge grid
    for n, approx in ((48, 368.0), (96, 184.0)):
        dt = cfl_dtb(grids(n), 5000.0)
        assert abs(dt / approx - 1.0) < 0.03


def test_w92_state(grids):
    g = grids(24)
    s = w92_case2_state(g)
    assert s["h0"].shape == (6, 30, 30)
    assert np.isfinite(s["ub"]).all()
