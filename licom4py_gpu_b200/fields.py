"""Initial states for the barotropic path.

* :func:`harmonic_state` -- seeded synthetic fields: a resting ocean of mean
  depth H with an SSH perturbation that is a sum of real spherical harmonics of
  degree 1..8 (all orders, N(0,1) coefficients, scaled to a target interior
  RMS), and lon/lat velocity components drawn the same way, rotated to
  covariant cubed-sphere components with ``a_l2c`` exactly as the reference's
  W92 initialiser does (src/licom/initial/w92_field.py:68-73).
* :func:`w92_case2_state` -- the reference's only physics scenario, Williamson
  (1992) case 2, following src/licom/initial/w92_field.py:36-96.
* :func:`cfl_dtb` -- barotropic step at a CFL number of the gravity-wave speed.

All fields are (6, M, M) float64 arrays on the host, evaluated at every point
including halos, like the reference (which evaluates W92 on the padded grid).
"""

from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np

HALO = 3
GRAV_CELERITY = 9.8     # src/licom/momentum/barotr_pure.py:24-25


def _legendre_all(lmax: int, x: np.ndarray) -> Dict[Tuple[int, int], np.ndarray]:
    """Fully normalised associated Legendre functions P_l^m(x), 0 <= m <= l <= lmax.

    Standard three-term recurrence in l at fixed m, seeded by the sectoral
    terms; normalised so that sum_m of the real harmonics is orthonormal on the
    unit sphere.
    """
    out: Dict[Tuple[int, int], np.ndarray] = {}
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    pmm = np.ones_like(x) * math.sqrt(1.0 / (4.0 * math.pi))
    for m in range(0, lmax + 1):
        if m > 0:
            pmm = -math.sqrt((2.0 * m + 1.0) / (2.0 * m)) * s * pmm
        out[(m, m)] = pmm
        if m + 1 <= lmax:
            p1 = math.sqrt(2.0 * m + 3.0) * x * pmm
            out[(m + 1, m)] = p1
            pl2, pl1 = pmm, p1
            for l in range(m + 2, lmax + 1):
                a = math.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
                b = math.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
                pl = a * (x * pl1 - b * pl2)
                out[(l, m)] = pl
                pl2, pl1 = pl1, pl
    return out


def harmonic_series(lon: np.ndarray, lat: np.ndarray, seed: int,
                    lmin: int = 1, lmax: int = 8) -> np.ndarray:
    """Sum of real spherical harmonics Y_lm, lmin <= l <= lmax, all m, N(0,1) coefficients.

    The coefficients are drawn from ``numpy.random.default_rng(seed)`` in the
    order l ascending, m = -l..l.
    """
    rng = np.random.default_rng(seed)
    ncoef = sum(2 * l + 1 for l in range(lmin, lmax + 1))
    coef = rng.standard_normal(ncoef)
    P = _legendre_all(lmax, np.sin(lat))
    field = np.zeros_like(lon, dtype=np.float64)
    k = 0
    for l in range(lmin, lmax + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            if m == 0:
                y = P[(l, 0)]
            elif m > 0:
                y = math.sqrt(2.0) * P[(l, am)] * np.cos(am * lon)
            else:
                y = math.sqrt(2.0) * P[(l, am)] * np.sin(am * lon)
            field = field + coef[k] * y
            k += 1
    return field


def _interior(a: np.ndarray) -> np.ndarray:
    return a[:, HALO:-HALO, HALO:-HALO]


def _scale_rms(f: np.ndarray, rms: float) -> np.ndarray:
    cur = math.sqrt(float(np.mean(_interior(f) ** 2)))
    return f * (rms / cur) if cur > 0 else f


def harmonic_state(grid: Dict[str, np.ndarray], seed: int, h_rms: float = 1.0,
                   uv_rms: float = 0.3) -> Dict[str, np.ndarray]:
    """Seeded (h0, ub, vb) on the padded grid; h0 is the perturbation about the mean depth.

    ``grid`` needs ``a_pt`` (6, M, M, 2) lon/lat and ``a_l2c`` (6, M, M, 2, 2).
    The h series uses ``seed``, the lon/lat velocity series ``seed+1`` and
    ``seed+2``; RMS values are measured over the interior cells.
    """
    lon = grid["a_pt"][..., 0]
    lat = grid["a_pt"][..., 1]
    h = _scale_rms(harmonic_series(lon, lat, seed), h_rms)
    ul = harmonic_series(lon, lat, seed + 1)
    vl = harmonic_series(lon, lat, seed + 2)
    spd = math.sqrt(float(np.mean(_interior(ul) ** 2 + vl[:, HALO:-HALO, HALO:-HALO] ** 2)) / 2.0)
    if spd > 0:
        ul = ul * (uv_rms / spd)
        vl = vl * (uv_rms / spd)
    l2c = grid["a_l2c"]
    ub = l2c[..., 0, 0] * ul + l2c[..., 0, 1] * vl
    vb = l2c[..., 1, 0] * ul + l2c[..., 1, 1] * vl
    return {"h0": h, "ub": ub, "vb": vb}


def w92_case2_state(grid: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """Williamson-1992 case 2 steady geostrophic flow (src/licom/initial/w92_field.py:36-96)."""
    lon = grid["a_pt"][..., 0]
    lat = grid["a_pt"][..., 1]
    l2c = grid["a_l2c"]
    ubar, alpha, radius, omega, grav = 1.0, 0.0, 6.371e6, 7.292e-5, 9.80
    u_lon = ubar * (np.cos(alpha) * np.cos(lat) + np.sin(alpha) * np.cos(lon) * np.sin(lat))
    u_lat = -ubar * np.sin(alpha) * np.sin(lon)
    ub = l2c[..., 0, 0] * u_lon + l2c[..., 0, 1] * u_lat
    vb = l2c[..., 1, 0] * u_lon + l2c[..., 1, 1] * u_lat
    h0 = (-(radius * omega * ubar + ubar ** 2 / 2.0)
          * ((-np.cos(lon) * np.cos(lat) * np.sin(alpha) + np.sin(lat) * np.cos(alpha)) ** 2
             - 1.0 / 3.0) / grav)
    return {"h0": h0, "ub": ub, "vb": vb}


def cfl_dtb(grid: Dict[str, np.ndarray], depth: float, cfl: float = 0.5) -> float:
    """dtb = cfl * min interior (dx, dy) / sqrt(g H); dx, dy from 1/rdx, 1/rdy."""
    dx = 1.0 / _interior(grid["rdx"])
    dy = 1.0 / _interior(grid["rdy"])
    return float(cfl * min(dx.min(), dy.min()) / math.sqrt(GRAV_CELERITY * depth))
