"""CPU float64 oracle of the LICOM barotropic RK2/RK3 path on the cubed-sphere duogrid.

TEST INFRASTRUCTURE: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` import this module, and only as the checker or
the timed CPU baseline.  The package never imports it; the GPU path has no CPU
fallback.

This is an independent NumPy restatement of the reference algorithm (it does
not import the reference).  It is pinned against golden vectors produced by
running the reference's own source (``tests/golden/make_golden.py``), and the
tests check it reproduces them bit for bit.

Arrays are (6, M, M) float64, M = N + 6; axis -2 is the Fortran i index
("x": rdx, ub_cx), axis -1 the Fortran j index ("y": rdy, vb_cy).  Interior
cells are 3..M-4 on both axes.  Each function cites the reference lines it
restates (paths within the reference project).
"""

from __future__ import annotations

from typing import Sequence, Tuple

import numpy as np

H = 3  # halo width, src/licom/kernel/cube.py:26

# 3rd-order reconstruction coefficients, src/licom/operators/poly.py:29-37
EP23, EP13, EP03, EM13, EM23 = -1.0 / 20.0, 9.0 / 20.0, 47.0 / 60.0, -13.0 / 60.0, 1.0 / 30.0
M13, M23, M33 = 37.0 / 60.0, -2.0 / 15.0, 1.0 / 60.0

E, W, N, S = 0, 1, 2, 3  # side ids, src/licom/kernel/communication.py:32


# --------------------------------------------------------------------------
# Stencil operators (full-array semantics, zero pads as in the reference)
# --------------------------------------------------------------------------
def _ax(a, axis, lo, hi):
    """a[..., lo:hi, :] (axis=-2) or a[..., lo:hi] (axis=-1)."""
    return a[..., lo:hi, :] if axis == -2 else a[..., lo:hi]


def _put(out, axis, lo, hi, val):
    if axis == -2:
        out[..., lo:hi, :] = val
    else:
        out[..., lo:hi] = val


def face_recon(a, axis):
    """5-point upwind-biased face values (east/west or north/south) along ``axis``.

    poly.py:39-93: valid for index 2..M-3, zero elsewhere.
    Returns (plus, minus) = (value at the + face of cell i, value at the - face of cell i).
    """
    m = a.shape[axis]
    t0, t1, t2, t3, t4 = (_ax(a, axis, k, m - 4 + k) for k in range(5))
    plus = EM23 * t0 + EM13 * t1 + EP03 * t2 + EP13 * t3 + EP23 * t4
    minus = EP23 * t0 + EP13 * t1 + EP03 * t2 + EM13 * t3 + EM23 * t4
    p = np.zeros_like(a)
    q = np.zeros_like(a)
    _put(p, axis, 2, m - 2, plus)
    _put(q, axis, 2, m - 2, minus)
    return p, q


def mid_value(a, axis):
    """6-point centred value at the - face of cell i along ``axis`` (poly.py:109-145).

    Valid for i in 3..M-3 along ``axis`` and 3..M-3 along the other axis, zero elsewhere.
    """
    m = a.shape[-1]
    if axis == -2:
        c = a[..., :, 3:m - 2]
        r = lambda k: c[..., k:m - 5 + k, :]  # noqa: E731
        core = M13 * (r(2) + r(3)) + M23 * (r(1) + r(4)) + M33 * (r(0) + r(5))
        out = np.zeros_like(a)
        out[..., 3:m - 2, 3:m - 2] = core
    else:
        c = a[..., 3:m - 2, :]
        r = lambda k: c[..., k:m - 5 + k]  # noqa: E731
        core = M13 * (r(2) + r(3)) + M23 * (r(1) + r(4)) + M33 * (r(0) + r(5))
        out = np.zeros_like(a)
        out[..., 3:m - 2, 3:m - 2] = core
    return out


def celerity(h, dzph_x, dzph_y):
    """barotr_pure.py:21-26"""
    cx = np.sqrt(9.8 * (mid_value(h, -2) + dzph_x))
    cy = np.sqrt(9.8 * (mid_value(h, -1) + dzph_y))
    return np.maximum(cx, 10.0), np.maximum(cy, 10.0)


def to_contravariant(u, v, gct, sina):
    """remap.py:34-39"""
    uct = (gct[..., 0, 0] * u + gct[..., 0, 1] * v) * sina
    vct = (gct[..., 1, 0] * u + gct[..., 1, 1] * v) * sina
    return uct, vct


def c_grid_normal(uct, vct):
    """remap.py:41-55: ub_cx[i] = (ue[i-1] + uw[i]) / 2 on axis -2, vb_cy on axis -1, i in 3..M-3."""
    m = uct.shape[-1]
    ue, uw = face_recon(uct, -2)
    vn, vs = face_recon(vct, -1)
    ucx = np.zeros_like(uct)
    vcy = np.zeros_like(vct)
    ucx[..., 3:m - 2, :] = 0.5 * (ue[..., 2:m - 3, :] + uw[..., 3:m - 2, :])
    vcy[..., 3:m - 2] = 0.5 * (vn[..., 2:m - 3] + vs[..., 3:m - 2])
    return ucx, vcy


def d_grid_upwind(u, v, ucx, vcy):
    """remap.py:73-95: tangential components by upwind selection on the normal component."""
    m = u.shape[-1]
    un, us = face_recon(u, -1)
    ve, vw = face_recon(v, -2)
    vcx = np.zeros_like(v)
    vcx[..., 3:m - 2, :] = np.where(ucx[..., 3:m - 2, :] > 0.0, ve[..., 2:m - 3, :], vw[..., 3:m - 2, :])
    ucy = np.zeros_like(u)
    ucy[..., 3:m - 2] = np.where(vcy[..., 3:m - 2] > 0.0, un[..., 2:m - 3], us[..., 3:m - 2])
    return ucy, vcx


def velocity_viscosity(cx, cy, h, ucx, vcy):
    """barotr_pure.py:29-34"""
    m = h.shape[-1]
    he, hw = face_recon(h, -2)
    hn, hs = face_recon(h, -1)
    ucx = ucx.copy()
    vcy = vcy.copy()
    ucx[..., 3:m - 2, :] += 4.9 / cx[..., 3:m - 2, :] * (he[..., 2:m - 3, :] - hw[..., 3:m - 2, :])
    vcy[..., 3:m - 2] += 4.9 / cy[..., 3:m - 2] * (hn[..., 2:m - 3] - hs[..., 3:m - 2])
    return ucx, vcy


def mass_flux(h, ucx, vcy, dzph_x, dzph_y):
    """barotr_pure.py:37-49"""
    he, hw = face_recon(h, -2)
    hn, hs = face_recon(h, -1)
    fu = dzph_x * ucx
    fv = dzph_y * vcy
    fu[..., 1:, :] += np.where(ucx[..., 1:, :] > 0.0, he[..., :-1, :], hw[..., 1:, :]) * ucx[..., 1:, :]
    fv[..., 1:] += np.where(vcy[..., 1:] > 0.0, hn[..., :-1], hs[..., 1:]) * vcy[..., 1:]
    return fu, fv


def divergence(fu, fv, rda, c_dy, d_dx):
    """agrid.py:43-53"""
    out = np.zeros_like(fu)
    out[..., :-1, :-1] = rda[..., :-1, :-1] * (
        fu[..., 1:, :-1] * c_dy[..., 1:, :-1] - fu[..., :-1, :-1] * c_dy[..., :-1, :-1]
        + fv[..., :-1, 1:] * d_dx[..., :-1, 1:] - fv[..., :-1, :-1] * d_dx[..., :-1, :-1])
    return out


def vorticity(vcx, ucy, rda, d_dx, c_dy):
    """agrid.py:31-41"""
    out = np.zeros_like(vcx)
    out[..., :-1, :-1] = rda[..., :-1, :-1] * (
        ucy[..., :-1, :-1] * d_dx[..., :-1, :-1] + vcx[..., 1:, :-1] * c_dy[..., 1:, :-1]
        - ucy[..., :-1, 1:] * d_dx[..., :-1, 1:] - vcx[..., :-1, :-1] * c_dy[..., :-1, :-1])
    return out


def advection(vcx, ucy, ucx, vcy, vct, uct, rdx, rdy, rda, d_dx, c_dy):
    """barotr_pure.py:78-97"""
    vort = vorticity(vcx, ucy, rda, d_dx, c_dy)
    ku = 0.5 * (ucx ** 2 + vcx ** 2)
    kv = 0.5 * (vcy ** 2 + ucy ** 2)
    advx = np.zeros_like(vcx)
    advy = np.zeros_like(vcx)
    advx[..., :-1, :] = vort[..., :-1, :] * vct[..., :-1, :] - (ku[..., 1:, :] - ku[..., :-1, :]) * rdx[..., :-1, :]
    advy[..., :-1] = -vort[..., :-1] * uct[..., :-1] - (kv[..., 1:] - kv[..., :-1]) * rdy[..., :-1]
    return advx, advy


def pgf_viscosity(cx, cy, rdx, rdy, uct, vct):
    """barotr_pure.py:63-75"""
    m = uct.shape[-1]
    ue, uw = face_recon(uct, -2)
    vn, vs = face_recon(vct, -1)
    fx = 0.5 * cx[..., 3:m - 2, :] * (ue[..., 2:m - 3, :] - uw[..., 3:m - 2, :])   # x faces 3..M-3
    fy = 0.5 * cy[..., 3:m - 2] * (vn[..., 2:m - 3] - vs[..., 3:m - 2])             # y faces 3..M-3
    visx = np.zeros_like(uct)
    visy = np.zeros_like(uct)
    visx[..., 3:m - 3, 3:m - 3] = -(rdx[..., 3:m - 3, 3:m - 3] * (fx[..., 1:, 3:m - 3] - fx[..., :-1, 3:m - 3]))
    visy[..., 3:m - 3, 3:m - 3] = -(rdy[..., 3:m - 3, 3:m - 3] * (fy[..., 3:m - 3, 1:] - fy[..., 3:m - 3, :-1]))
    return visx, visy


def pressure_gradient(h, rdx, rdy):
    """barotr_pure.py:57-60 with agrid.py:55-69"""
    m = h.shape[-1]
    hx = mid_value(h, -2)
    hy = mid_value(h, -1)
    gx = np.zeros_like(h)
    gy = np.zeros_like(h)
    gx[..., 3:m - 3, 3:m - 3] = rdx[..., 3:m - 3, 3:m - 3] * (hx[..., 4:m - 2, 3:m - 3] - hx[..., 3:m - 3, 3:m - 3])
    gy[..., 3:m - 3, 3:m - 3] = rdy[..., 3:m - 3, 3:m - 3] * (hy[..., 3:m - 3, 4:m - 2] - hy[..., 3:m - 3, 3:m - 3])
    return -9.80 * gx, -9.80 * gy


# --------------------------------------------------------------------------
# Cubed-sphere connectivity and the duogrid halo
# --------------------------------------------------------------------------
def face_neighbor(t: int, d: int) -> Tuple[int, int, bool]:
    """(neighbour face, its side, reversed) for side d of face t (0-based faces).

    Adjacency of communication.py:57-87 (even/odd face rules); the join of an
    E/W side with an S/N side reverses the along-edge index
    (communication.py:41-55, FLIP_I_TRANS); E-W and N-S joins keep it.
    """
    if t % 2 == 0:
        rules = {S: ((t + 4) % 6, E), E: ((t + 2) % 6, S), N: ((t + 1) % 6, S), W: ((t + 5) % 6, E)}
    else:
        rules = {E: ((t + 1) % 6, W), N: ((t + 2) % 6, W), W: ((t + 4) % 6, N), S: ((t + 5) % 6, N)}
    nb, side = rules[d]
    rev = (d in (E, W)) != (side in (E, W))
    return nb, side, rev


def _interior_lines(a, f, side, m):
    """The three interior lines of face f nearest ``side``, as [c, k] (c = 0..2, k along the edge).

    Line order follows the packing of communication.py:193-207.
    """
    n = m - 2 * H
    if side == E:
        return a[f, H:H + n, m - 2 * H:m - H].T
    if side == W:
        return a[f, H:H + n, H:2 * H].T
    if side == N:
        return a[f, m - 2 * H:m - H, H:H + n]
    return a[f, H:2 * H, H:H + n]


def copy_halo(a):
    """Halo copy from the neighbouring faces without corners (communication.py:387-474, px=py=1)."""
    out = a.copy()
    m = a.shape[-1]
    n = m - 2 * H
    for t in range(6):
        for d in (E, W, N, S):
            nb, side, rev = face_neighbor(t, d)
            q = _interior_lines(a, nb, side, m)
            if rev:
                q = q[:, ::-1]
            if d == E:
                out[t, H:H + n, m - H:] = q.T
            elif d == W:
                out[t, H:H + n, :H] = q.T
            elif d == N:
                out[t, m - H:, H:H + n] = q
            else:
                out[t, :H, H:H + n] = q
    return out


def kik_to_ext(a, coef, loc_i, loc_j):
    """Linear kinked->extended interpolation along each halo band, then corners (cube.py:40-127)."""
    out = a.copy()
    m = a.shape[-1]
    f = np.arange(6)[:, None, None]
    c = np.arange(H)[None, None, :]
    # W and E bands: interpolate along axis -2 inside the band columns
    for cols in (slice(0, H), slice(m - H, m)):
        band = a[:, :, cols]
        loc = loc_i[:, H:m - H, cols]
        w = coef[:, H:m - H, cols]
        out[:, H:m - H, cols] = w[..., 0] * band[f, loc, c] + w[..., 1] * band[f, loc + 1, c]
    r = np.arange(H)[None, :, None]
    for rows in (slice(0, H), slice(m - H, m)):
        band = a[:, rows, :]
        loc = loc_j[:, rows, H:m - H]
        w = coef[:, rows, H:m - H]
        out[:, rows, H:m - H] = w[..., 0] * band[f, r, loc] + w[..., 1] * band[f, r, loc + 1]
    sw, se = out[:, H, :H].copy(), out[:, H, m - H:].copy()
    nw, ne = out[:, m - H - 1, :H].copy(), out[:, m - H - 1, m - H:].copy()
    out[:, :H, :H] = sw[:, None, :]
    out[:, :H, m - H:] = se[:, None, :]
    out[:, m - H:, :H] = nw[:, None, :]
    out[:, m - H:, m - H:] = ne[:, None, :]
    return out


def fill_scalar(a, coef, loc_i, loc_j):
    """ext_scalar, cube.py:130-134"""
    return kik_to_ext(copy_halo(a), coef, loc_i, loc_j)


def fill_vector(u, v, coef, loc_i, loc_j, c2l, l2c, inner, outer):
    """ext_vector, cube.py:137-153"""
    ull = (c2l[..., 0, 0] * u + c2l[..., 0, 1] * v) * inner
    vll = (c2l[..., 1, 0] * u + c2l[..., 1, 1] * v) * inner
    ull = fill_scalar(ull, coef, loc_i, loc_j)
    vll = fill_scalar(vll, coef, loc_i, loc_j)
    un = (l2c[..., 0, 0] * ull + l2c[..., 0, 1] * vll) * outer + u * inner
    vn = (l2c[..., 1, 0] * ull + l2c[..., 1, 1] * vll) * outer + v * inner
    return un, vn


def _edge_line(u, v, f, side, m):
    """Face-normal C-grid line on ``side`` of face f (communication.py:226-235, 247-251)."""
    n = m - 2 * H
    if side == E:
        return v[f, H:H + n, m - H]
    if side == W:
        return v[f, H:H + n, H]
    if side == N:
        return u[f, m - H, H:H + n]
    return u[f, H, H:H + n]


def edge_average(u, v):
    """boundary_communication (communication.py:504-570): mean of the two faces' normal values."""
    m = u.shape[-1]
    n = m - 2 * H
    uo, vo = u.copy(), v.copy()
    for t in range(6):
        for d in (E, W, N, S):
            nb, side, rev = face_neighbor(t, d)
            other = _edge_line(u, v, nb, side, m)
            if rev:
                other = other[::-1]
            own = _edge_line(u, v, t, d, m)
            val = (own + other) / 2.0
            if d == E:
                vo[t, H:H + n, m - H] = val
            elif d == W:
                vo[t, H:H + n, H] = val
            elif d == N:
                uo[t, m - H, H:H + n] = val
            else:
                uo[t, H, H:H + n] = val
    return uo, vo


# --------------------------------------------------------------------------
# One RK stage and the substep loops
# --------------------------------------------------------------------------
def stage(h0, h0p, ub, vb, ubp, vbp, consts: Sequence[np.ndarray], dt: float, beta: float,
          last: bool):
    """One RK stage, barotr_pure.py:100-168.  Returns the 13 stage outputs."""
    (dzph_x, dzph_y, rdx, rdy, a_f, coef, loc_i, loc_j, c2l, l2c, inner, outer,
     gct, sina, rda, c_dy, d_dx) = consts[:17]
    cx, cy = celerity(h0, dzph_x, dzph_y)
    uct, vct = to_contravariant(ub, vb, gct, sina)
    ucx, vcy = c_grid_normal(uct, vct)
    ucx, vcy = edge_average(ucx, vcy)
    ucy, vcx = d_grid_upwind(ub, vb, ucx, vcy)
    ucx, vcy = velocity_viscosity(cx, cy, h0, ucx, vcy)
    fu, fv = mass_flux(h0, ucx, vcy, dzph_x, dzph_y)
    if last:
        fu, fv = edge_average(fu, fv)
    hn = h0p - divergence(fu, fv, rda, c_dy, d_dx) * dt
    hn = fill_scalar(hn, coef, loc_i, loc_j)
    advx, advy = advection(vcx, ucy, ucx, vcy, vct, uct, rdx, rdy, rda, d_dx, c_dy)
    visx, visy = pgf_viscosity(cx, cy, rdx, rdy, uct, vct)
    hb = (1.0 - beta) * hn + beta * h0
    pu, pv = pressure_gradient(hb, rdx, rdy)
    un = ubp + (pu + advx + a_f * vct + visx) * dt
    vn = vbp + (pv + advy - a_f * uct + visy) * dt
    un, vn = fill_vector(un, vn, coef, loc_i, loc_j, c2l, l2c, inner, outer)
    return (hn, un, vn, cx, cy, uct, vct, ucx, ucy, vcx, vcy, advx, advy)


def rk2_core(state: Sequence[np.ndarray], consts: Sequence[np.ndarray], nbb: int, dtb: float):
    """_barotr_rk2_core, barotr.py:41-61: midpoint RK2 (dt/2 then dt from the same base)."""
    st = tuple(state)
    coupling = st[16:23]
    for _ in range(nbb):
        h0, h0p, ub, vb, ubp, vbp = st[:6]
        r1 = stage(h0, h0p, ub, vb, ubp, vbp, consts, dtb / 2.0, 0.0, False)
        r2 = stage(r1[0], h0p, r1[1], r1[2], ubp, vbp, consts, dtb, 0.0, True)
        st = (r2[0], r2[0], r2[1], r2[2], r2[1], r2[2], *r2[3:]) + tuple(coupling)
    return st


def rk3_core(state: Sequence[np.ndarray], consts: Sequence[np.ndarray], nbb: int, dtb: float):
    """_barotr_rk3_core, barotr.py:64-87: dt/3, dt/2, dt with beta_d = 1."""
    st = tuple(state)
    coupling = st[16:23]
    for _ in range(nbb):
        h0, h0p, ub, vb, ubp, vbp = st[:6]
        r1 = stage(h0, h0p, ub, vb, ubp, vbp, consts, dtb / 3.0, 1.0, False)
        r2 = stage(r1[0], h0p, r1[1], r1[2], ubp, vbp, consts, dtb / 2.0, 1.0, False)
        r3 = stage(r2[0], h0p, r2[1], r2[2], ubp, vbp, consts, dtb, 1.0, True)
        st = (r3[0], r3[0], r3[1], r3[2], r3[1], r3[2], *r3[3:]) + tuple(coupling)
    return st


def interior(a):
    return a[..., H:-H, H:-H]
