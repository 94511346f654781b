// bt_stencil.cuh - device functions of the barotropic RK stage on the duogrid.
//
// One RK stage (src/licom/momentum/barotr_pure.py:100-168) is split at its two
// global dependencies into two tile phases:
//
//   phase H  (tile_h):  celerity, A->C remap, C-grid edge average, D-grid
//            upwind, velocity viscosity, mass flux (+ flux edge average on
//            the last stage), divergence, new h = h_base - div*dt.
//   phase UV (tile_uv): the same C/D-grid face quantities recomputed from the
//            stage input, vorticity/kinetic-energy advection, celerity
//            viscosity, pressure gradient of the new h, momentum update.
//
// The ext_scalar / ext_vector halo fills of the reference (cube.py:130-153)
// become gathers done by whoever reads a halo cell (fetch_s / fetch_v), and
// the boundary_communication edge averages (communication.py:504-570) are
// computed in place by recomputing the neighbouring face's edge value from
// that face's data (nb_normal_raw / nb_mass_flux).
//
// Every arithmetic expression keeps the reference's operand order; with
// -fmad=false the float64 instantiation rounds exactly like the NumPy run of
// the reference.

#pragma once

#include "bt_common.cuh"

namespace bt {

// 3rd-order reconstruction coefficients, src/licom/operators/poly.py:29-37
#define BT_EP23 (-1.0 / 20.0)
#define BT_EP13 (9.0 / 20.0)
#define BT_EP03 (47.0 / 60.0)
#define BT_EM13 (-13.0 / 60.0)
#define BT_EM23 (1.0 / 30.0)
#define BT_M13 (37.0 / 60.0)
#define BT_M23 (-2.0 / 15.0)
#define BT_M33 (1.0 / 60.0)

// Value at the + face of the centre point of p[0], p[s], .., p[4s] (poly.py:50-56)
template <typename T>
__device__ __forceinline__ T rplus(const T* p, int s) {
  return T(BT_EM23) * p[0] + T(BT_EM13) * p[s] + T(BT_EP03) * p[2 * s] + T(BT_EP13) * p[3 * s] +
         T(BT_EP23) * p[4 * s];
}
// Value at the - face of the centre point (poly.py:57-63)
template <typename T>
__device__ __forceinline__ T rminus(const T* p, int s) {
  return T(BT_EP23) * p[0] + T(BT_EP13) * p[s] + T(BT_EP03) * p[2 * s] + T(BT_EM13) * p[3 * s] +
         T(BT_EM23) * p[4 * s];
}
// 6-point centred face value between p[2s] and p[3s] (poly.py:120-124)
template <typename T>
__device__ __forceinline__ T mid6(const T* p, int s) {
  return T(BT_M13) * (p[2 * s] + p[3 * s]) + T(BT_M23) * (p[s] + p[4 * s]) +
         T(BT_M33) * (p[0] + p[5 * s]);
}
// Gravity-wave speed with the 10 m/s floor (barotr_pure.py:21-26); NaN propagates like jnp.maximum.
template <typename T>
__device__ __forceinline__ T celerity(T hface, T dz) {
  T c = sqrt(T(9.8) * (hface + dz));
  return (c < T(10.0)) ? T(10.0) : c;
}

// ---------------------------------------------------------------------------
// Halo values on the fly
// ---------------------------------------------------------------------------
// Scalar value at (f, i, j).  Interior cells (and every cell when the stored
// halo is valid) are read directly; a halo cell is the kinked->extended linear
// interpolation of two interior cells of a neighbouring face (cube.py:40-134).
template <typename T>
__device__ __forceinline__ T fetch_s(const T* F, const Geo<T>& g, int f, int i, int j, int stored) {
  const int m = g.m;
  if (stored || is_interior(i, j, m)) return F[cell(f, i, j, m)];
  const int k = f * g.nh + halo_id(i, j, m);
  const int2 s = g.hsrc[k];
  const T w0 = g.hw[2 * k], w1 = g.hw[2 * k + 1];
  return w0 * F[s.x] + w1 * F[s.y];
}

// Vector (covariant u, v) at (f, i, j): the halo value is rotated to lon/lat at
// the two source cells with c2l, interpolated, and rotated back with the
// target's l2c (ext_vector, cube.py:137-153; the inner/outer masks are 1/0 there).
template <typename T>
__device__ __forceinline__ void fetch_v(const T* U, const T* V, const Geo<T>& g, int f, int i, int j,
                                        int stored, T& u, T& v) {
  const int m = g.m;
  const long o = cell(f, i, j, m);
  if (stored || is_interior(i, j, m)) {
    u = U[o];
    v = V[o];
    return;
  }
  const int k = f * g.nh + halo_id(i, j, m);
  const int2 s = g.hsrc[k];
  const T w0 = g.hw[2 * k], w1 = g.hw[2 * k + 1];
  const T* C0 = g.c2l + 4 * (long)s.x;
  const T* C1 = g.c2l + 4 * (long)s.y;
  const T u0 = U[s.x], v0 = V[s.x], u1 = U[s.y], v1 = V[s.y];
  const T ull0 = C0[0] * u0 + C0[1] * v0, vll0 = C0[2] * u0 + C0[3] * v0;
  const T ull1 = C1[0] * u1 + C1[1] * v1, vll1 = C1[2] * u1 + C1[3] * v1;
  const T ull = w0 * ull0 + w1 * ull1;
  const T vll = w0 * vll0 + w1 * vll1;
  const T* L = g.l2c + 4 * o;
  u = L[0] * ull + L[1] * vll;
  v = L[2] * ull + L[3] * vll;
}

// Contravariant component along axis -2 (x) or axis -1 (y) (remap.py:34-39)
template <typename T>
__device__ __forceinline__ T contra(const Geo<T>& g, long o, T u, T v, int y) {
  const T* G = g.gct + 4 * o;
  return y ? (G[2] * u + G[3] * v) * g.sina[o] : (G[0] * u + G[1] * v) * g.sina[o];
}

// ---------------------------------------------------------------------------
// The neighbouring face's side of a C-grid edge
// ---------------------------------------------------------------------------
// k-th of the 6 points (k = 0..5) on the line normal to ``side`` of a face that
// straddles that side's C-grid edge face, at along-edge position kk.  The
// edge face itself sits between points 2 and 3.
__device__ __forceinline__ void edge_point(int side, int kk, int k, int m, int& i, int& j) {
  switch (side) {
    case kS: i = k; j = kHalo + kk; break;
    case kN: i = m - 6 + k; j = kHalo + kk; break;
    case kW: i = kHalo + kk; j = k; break;
    default: i = kHalo + kk; j = m - 6 + k; break;
  }
}

// The neighbour's C-grid normal velocity before averaging, at the edge shared
// with side ``side`` of face f, position k along our edge
// (communication.py:226-235 pack + remap.py:41-55 on the neighbour).
template <typename T>
__device__ T nb_normal_raw(const Geo<T>& g, const T* U, const T* V, int stored, int f, int side,
                           int k) {
  const int r = g.route[f * 4 + side];
  const int nb = route_nb(r), ns = route_side(r);
  const int kk = route_rev(r) ? g.n - 1 - k : k;
  const int y = (ns == kE || ns == kW);
  T p[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    int i, j;
    edge_point(ns, kk, q, g.m, i, j);
    T u, v;
    fetch_v(U, V, g, nb, i, j, stored, u, v);
    p[q] = contra(g, cell(nb, i, j, g.m), u, v, y);
  }
  return T(0.5) * (rplus(p, 1) + rminus(p + 1, 1));
}

// The neighbour's mass flux at the shared edge on the last stage, given the
// (already averaged, hence common) edge velocity ``bc`` (barotr_pure.py:29-49
// evaluated on the neighbour, then communication.py:504-570 on the fluxes).
template <typename T>
__device__ T nb_mass_flux(const Geo<T>& g, const T* H, int stored, int f, int side, int k, T bc) {
  const int r = g.route[f * 4 + side];
  const int nb = route_nb(r), ns = route_side(r);
  const int kk = route_rev(r) ? g.n - 1 - k : k;
  const int y = (ns == kE || ns == kW);
  T p[6];
  int fi = 0, fj = 0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    int i, j;
    edge_point(ns, kk, q, g.m, i, j);
    if (q == 3) {
      fi = i;
      fj = j;
    }
    p[q] = fetch_s(H, g, nb, i, j, stored);
  }
  const long o = cell(nb, fi, fj, g.m);
  const T dz = y ? g.dzph_y[o] : g.dzph_x[o];
  const T he = rplus(p, 1), hw = rminus(p + 1, 1);
  const T c = celerity(mid6(p, 1), dz);
  const T vis = bc + (T(4.9) / c) * (he - hw);
  return dz * vis + (vis > T(0.0) ? he : hw) * vis;
}

// Side of a face whose C-grid edge lies at x-face index i (or y-face index j).
__device__ __forceinline__ int xface_side(int i, int m) {
  return i == kHalo ? kS : (i == m - kHalo ? kN : -1);
}
__device__ __forceinline__ int yface_side(int j, int m) {
  return j == kHalo ? kW : (j == m - kHalo ? kE : -1);
}

// ---------------------------------------------------------------------------
// Tile phases
// ---------------------------------------------------------------------------
template <int TI, int TJ>
struct TileShape {
  static constexpr int RI = TI + 6, RJ = TJ + 6, R = RI * RJ;
  static constexpr int FX = (TI + 1) * TJ;   // x faces
  static constexpr int FY = TI * (TJ + 1);   // y faces
  static constexpr int kWordsH = 3 * R + FX + FY;
  static constexpr int kWordsUV = 6 * R + 3 * FX + 3 * FY;
};

struct TileBox {
  int f, i0, j0, ni, nj;
};

__device__ __forceinline__ TileBox tile_box(const Tiling& t, int n, int tile) {
  TileBox b;
  const int per_face = t.nti * t.ntj;
  b.f = tile / per_face;
  const int r = tile - b.f * per_face;
  const int ti = r / t.ntj, tj = r - ti * t.ntj;
  b.i0 = kHalo + ti * t.ti;
  b.j0 = kHalo + tj * t.tj;
  b.ni = min(t.ti, n - ti * t.ti);
  b.nj = min(t.tj, n - tj * t.tj);
  return b;
}

// Region point (r, c) of a tile's smem block is needed when it lies in the
// tile's rows or columns, extended by 3 along the other axis (no region corners).
__device__ __forceinline__ bool region_needed(int r, int c, int ni, int nj) {
  const bool rin = r >= kHalo && r < kHalo + ni, cin = c >= kHalo && c < kHalo + nj;
  return (rin && c < nj + 6) || (cin && r < ni + 6);
}

// Phase H of one tile: writes the new h on the tile's interior cells.
template <typename T, int TI, int TJ>
__device__ void tile_h(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm) {
  using S = TileShape<TI, TJ>;
  constexpr int RJ = S::RJ;
  const int m = g.m, f = b.f;
  T* s_h = sm;
  T* s_uc = s_h + S::R;
  T* s_vc = s_uc + S::R;
  T* s_fu = s_vc + S::R;  // [TI+1][TJ]
  T* s_fv = s_fu + S::FX; // [TI][TJ+1]

  for (int e = threadIdx.x; e < S::R; e += blockDim.x) {
    const int r = e / RJ, c = e - r * RJ;
    if (!region_needed(r, c, b.ni, b.nj)) continue;
    const int i = b.i0 - kHalo + r, j = b.j0 - kHalo + c;
    const long o = cell(f, i, j, m);
    T u, v;
    fetch_v(io.u, io.v, g, f, i, j, io.stored_halo, u, v);
    s_h[e] = fetch_s(io.h, g, f, i, j, io.stored_halo);
    s_uc[e] = contra(g, o, u, v, 0);
    s_vc[e] = contra(g, o, u, v, 1);
  }
  __syncthreads();

  // x faces i = i0 .. i0+ni, columns of the tile
  for (int e = threadIdx.x; e < (b.ni + 1) * b.nj; e += blockDim.x) {
    const int a = e / b.nj, q = e - a * b.nj;
    const int i = b.i0 + a, j = b.j0 + q;
    const int base = a * RJ + (q + kHalo);  // local (row of cell i) - 3
    const T* ph = s_h + base;
    const T* pu = s_uc + base;
    const T ue = rplus(pu, RJ), uw = rminus(pu + RJ, RJ);
    T bc = T(0.5) * (ue + uw);
    const int side = xface_side(i, m);
    if (side >= 0) bc = (bc + nb_normal_raw(g, io.u, io.v, io.stored_halo, f, side, j - kHalo)) / T(2.0);
    const long o = cell(f, i, j, m);
    const T dz = g.dzph_x[o];
    const T he = rplus(ph, RJ), hw = rminus(ph + RJ, RJ);
    const T cx = celerity(mid6(ph, RJ), dz);
    const T vis = bc + (T(4.9) / cx) * (he - hw);
    T fu = dz * vis + (vis > T(0.0) ? he : hw) * vis;
    if (io.last && side >= 0)
      fu = (fu + nb_mass_flux(g, io.h, io.stored_halo, f, side, j - kHalo, bc)) / T(2.0);
    s_fu[a * TJ + q] = fu;
  }
  // y faces j = j0 .. j0+nj, rows of the tile
  for (int e = threadIdx.x; e < b.ni * (b.nj + 1); e += blockDim.x) {
    const int a = e / (b.nj + 1), q = e - a * (b.nj + 1);
    const int i = b.i0 + a, j = b.j0 + q;
    const int base = (a + kHalo) * RJ + q;
    const T* ph = s_h + base;
    const T* pv = s_vc + base;
    const T vn = rplus(pv, 1), vs = rminus(pv + 1, 1);
    T bc = T(0.5) * (vn + vs);
    const int side = yface_side(j, m);
    if (side >= 0) bc = (bc + nb_normal_raw(g, io.u, io.v, io.stored_halo, f, side, i - kHalo)) / T(2.0);
    const long o = cell(f, i, j, m);
    const T dz = g.dzph_y[o];
    const T hn = rplus(ph, 1), hs = rminus(ph + 1, 1);
    const T cy = celerity(mid6(ph, 1), dz);
    const T vis = bc + (T(4.9) / cy) * (hn - hs);
    T fv = dz * vis + (vis > T(0.0) ? hn : hs) * vis;
    if (io.last && side >= 0)
      fv = (fv + nb_mass_flux(g, io.h, io.stored_halo, f, side, i - kHalo, bc)) / T(2.0);
    s_fv[a * (TJ + 1) + q] = fv;
  }
  __syncthreads();

  // cells: divergence (agrid.py:43-53) and the h update (barotr_pure.py:119-120)
  for (int e = threadIdx.x; e < b.ni * b.nj; e += blockDim.x) {
    const int a = e / b.nj, q = e - a * b.nj;
    const int i = b.i0 + a, j = b.j0 + q;
    const long o = cell(f, i, j, m);
    const T fu0 = s_fu[a * TJ + q], fu1 = s_fu[(a + 1) * TJ + q];
    const T fv0 = s_fv[a * (TJ + 1) + q], fv1 = s_fv[a * (TJ + 1) + q + 1];
    const T div = g.rda[o] * (fu1 * g.c_dy[o + m] - fu0 * g.c_dy[o] + fv1 * g.d_dx[o + 1] - fv0 * g.d_dx[o]);
    io.h_out[o] = io.hp[o] - div * io.dt;
  }
}

// Phase UV of one tile: writes the new u, v on the tile's interior cells.
// io.h_out must hold the new h of every face (interior) from phase H.
template <typename T, int TI, int TJ>
__device__ void tile_uv(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm) {
  using S = TileShape<TI, TJ>;
  constexpr int RJ = S::RJ;
  const int m = g.m, f = b.f;
  T* s_h = sm;
  T* s_uc = s_h + S::R;
  T* s_vc = s_uc + S::R;
  T* s_u = s_vc + S::R;
  T* s_v = s_u + S::R;
  T* s_hb = s_v + S::R;
  T* s_ku = s_hb + S::R;   // x faces [TI+1][TJ]: kinetic energy, tangential v, viscous flux
  T* s_vx = s_ku + S::FX;
  T* s_fx = s_vx + S::FX;
  T* s_kv = s_fx + S::FX;  // y faces [TI][TJ+1]
  T* s_uy = s_kv + S::FY;
  T* s_fy = s_uy + S::FY;

  for (int e = threadIdx.x; e < S::R; e += blockDim.x) {
    const int r = e / RJ, c = e - r * RJ;
    if (!region_needed(r, c, b.ni, b.nj)) continue;
    const int i = b.i0 - kHalo + r, j = b.j0 - kHalo + c;
    const long o = cell(f, i, j, m);
    T u, v;
    fetch_v(io.u, io.v, g, f, i, j, io.stored_halo, u, v);
    const T h = fetch_s(io.h, g, f, i, j, io.stored_halo);
    const T hn = fetch_s((const T*)io.h_out, g, f, i, j, 0);
    s_h[e] = h;
    s_u[e] = u;
    s_v[e] = v;
    s_uc[e] = contra(g, o, u, v, 0);
    s_vc[e] = contra(g, o, u, v, 1);
    s_hb[e] = (T(1.0) - io.beta) * hn + io.beta * h;  // fb_scheme, barotr_pure.py:52-54
  }
  __syncthreads();

  // x faces
  for (int e = threadIdx.x; e < (b.ni + 1) * b.nj; e += blockDim.x) {
    const int a = e / b.nj, q = e - a * b.nj;
    const int i = b.i0 + a, j = b.j0 + q;
    const int base = a * RJ + (q + kHalo);
    const T* ph = s_h + base;
    const T* pu = s_uc + base;
    const T* pv = s_v + base;
    const T ue = rplus(pu, RJ), uw = rminus(pu + RJ, RJ);
    T bc = T(0.5) * (ue + uw);
    const int side = xface_side(i, m);
    if (side >= 0) bc = (bc + nb_normal_raw(g, io.u, io.v, io.stored_halo, f, side, j - kHalo)) / T(2.0);
    const T vt = bc > T(0.0) ? rplus(pv, RJ) : rminus(pv + RJ, RJ);   // remap.py:84-88
    const long o = cell(f, i, j, m);
    const T cx = celerity(mid6(ph, RJ), g.dzph_x[o]);
    const T vis = bc + (T(4.9) / cx) * (rplus(ph, RJ) - rminus(ph + RJ, RJ));
    s_ku[a * TJ + q] = T(0.5) * (vis * vis + vt * vt);
    s_vx[a * TJ + q] = vt;
    s_fx[a * TJ + q] = T(0.5) * cx * (ue - uw);                       // barotr_pure.py:68
  }
  // y faces
  for (int e = threadIdx.x; e < b.ni * (b.nj + 1); e += blockDim.x) {
    const int a = e / (b.nj + 1), q = e - a * (b.nj + 1);
    const int i = b.i0 + a, j = b.j0 + q;
    const int base = (a + kHalo) * RJ + q;
    const T* ph = s_h + base;
    const T* pv = s_vc + base;
    const T* pu = s_u + base;
    const T vn = rplus(pv, 1), vs = rminus(pv + 1, 1);
    T bc = T(0.5) * (vn + vs);
    const int side = yface_side(j, m);
    if (side >= 0) bc = (bc + nb_normal_raw(g, io.u, io.v, io.stored_halo, f, side, i - kHalo)) / T(2.0);
    const T ut = bc > T(0.0) ? rplus(pu, 1) : rminus(pu + 1, 1);       // remap.py:90-94
    const long o = cell(f, i, j, m);
    const T cy = celerity(mid6(ph, 1), g.dzph_y[o]);
    const T vis = bc + (T(4.9) / cy) * (rplus(ph, 1) - rminus(ph + 1, 1));
    s_kv[a * (TJ + 1) + q] = T(0.5) * (vis * vis + ut * ut);
    s_uy[a * (TJ + 1) + q] = ut;
    s_fy[a * (TJ + 1) + q] = T(0.5) * cy * (vn - vs);                  // barotr_pure.py:69
  }
  __syncthreads();

  for (int e = threadIdx.x; e < b.ni * b.nj; e += blockDim.x) {
    const int a = e / b.nj, q = e - a * b.nj;
    const int i = b.i0 + a, j = b.j0 + q;
    const long o = cell(f, i, j, m);
    const int xf0 = a * TJ + q, xf1 = (a + 1) * TJ + q;
    const int yf0 = a * (TJ + 1) + q, yf1 = yf0 + 1;
    const int lc = (a + kHalo) * RJ + (q + kHalo);
    const T uct = s_uc[lc], vct = s_vc[lc];
    const T rdx = g.rdx[o], rdy = g.rdy[o];
    // vorticity (agrid.py:31-41) and advection (barotr_pure.py:78-97)
    const T vort = g.rda[o] * (s_uy[yf0] * g.d_dx[o] + s_vx[xf1] * g.c_dy[o + m] -
                               s_uy[yf1] * g.d_dx[o + 1] - s_vx[xf0] * g.c_dy[o]);
    const T advx = vort * vct - (s_ku[xf1] - s_ku[xf0]) * rdx;
    const T advy = -vort * uct - (s_kv[yf1] - s_kv[yf0]) * rdy;
    // celerity viscosity (barotr_pure.py:63-75)
    const T visx = -(rdx * (s_fx[xf1] - s_fx[xf0]));
    const T visy = -(rdy * (s_fy[yf1] - s_fy[yf0]));
    // pressure gradient of the new h (agrid.py:55-69, barotr_pure.py:57-60)
    const T* pbx = s_hb + (a * RJ + (q + kHalo));
    const T* pby = s_hb + ((a + kHalo) * RJ + q);
    const T pgu = T(-9.80) * (rdx * (mid6(pbx + RJ, RJ) - mid6(pbx, RJ)));
    const T pgv = T(-9.80) * (rdy * (mid6(pby + 1, 1) - mid6(pby, 1)));
    const T af = g.a_f[o];
    // momentum update (barotr_pure.py:149-150)
    io.u_out[o] = io.up[o] + (pgu + advx + af * vct + visx) * io.dt;
    io.v_out[o] = io.vp[o] + (pgv + advy - af * uct + visy) * io.dt;
  }
}

// ---------------------------------------------------------------------------
// Grid-wide barrier of the persistent round kernel
// ---------------------------------------------------------------------------
// Monotone arrival counter: the k-th barrier completes when the counter reaches
// k * gridDim.x.  Thread 0 of each CTA publishes the CTA's writes (fence), arrives
// and spins with a bounded number of polls; on timeout it raises
// kErrBarrierTimeout and every CTA leaves the round at its next barrier.
// Returns false when the round must stop.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned& gen, int* err, long long limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ++gen;
    const unsigned target = gen * gridDim.x;
    __threadfence();
    atomicAdd(bar, 1u);
    long long polls = 0;
    int ok = 1;
    while (true) {
      unsigned seen;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(bar) : "memory");
      if ((int)(seen - target) >= 0) break;
      if (++polls > limit) {
        atomicOr(err, kErrBarrierTimeout);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    if (ok && *((volatile int*)err) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Stage pointers of (substep, stage) of a round; mirrors the host schedule.
template <typename T>
__device__ StageIO<T> round_stage(const RoundArgs<T>& a, int step, int st) {
  StageIO<T> io;
  const T* const* cur = step == 0 ? a.x0 : (const T* const*)a.x;
  const T* const* base = step == 0 ? a.b0 : (const T* const*)a.x;
  const int nst = a.rk == 2 ? 2 : 3;
  const T* const* in = st == 0 ? cur : (st == 1 ? (const T* const*)a.y : (const T* const*)a.z);
  T* const* out = st == nst - 1 ? a.x : (st == 0 ? a.y : a.z);
  io.h = in[0];
  io.u = in[1];
  io.v = in[2];
  io.hp = base[0];
  io.up = base[1];
  io.vp = base[2];
  io.h_out = out[0];
  io.u_out = out[1];
  io.v_out = out[2];
  double dt;
  if (a.rk == 2) {
    dt = st == 0 ? a.dtb / 2.0 : a.dtb;      // barotr.py:50-56
    io.beta = T(0.0);
  } else {
    dt = st == 0 ? a.dtb / 3.0 : (st == 1 ? a.dtb / 2.0 : a.dtb);  // barotr.py:73-83
    io.beta = T(1.0);
  }
  io.dt = (T)dt;
  io.stored_halo = (step == 0 && st == 0) ? 1 : 0;
  io.last = st == nst - 1 ? 1 : 0;
  return io;
}

// ---------------------------------------------------------------------------
// Materialised halos (end of a round) and diagnostics
// ---------------------------------------------------------------------------
// Write every halo cell of face-major field(s) from their own interior.
template <typename T>
__device__ void fill_halo_cell(const Geo<T>& g, T* H, T* U, T* V, int k) {
  const int f = k / g.nh, id = k - f * g.nh;
  const int m = g.m, n = g.n;
  int i, j;
  if (id < 3 * m) {
    i = id / m;
    j = id - i * m;
  } else if (id < 6 * m) {
    i = m - kHalo + (id - 3 * m) / m;
    j = (id - 3 * m) % m;
  } else if (id < 6 * m + 3 * n) {
    i = kHalo + (id - 6 * m) / 3;
    j = (id - 6 * m) % 3;
  } else {
    i = kHalo + (id - 6 * m - 3 * n) / 3;
    j = m - kHalo + (id - 6 * m - 3 * n) % 3;
  }
  const long o = cell(f, i, j, m);
  if (H) H[o] = fetch_s(H, g, f, i, j, 0);
  if (U) {
    T u, v;
    fetch_v(U, V, g, f, i, j, 0, u, v);
    U[o] = u;
    V[o] = v;
  }
}

template <typename T>
struct DiagOut {
  T* cx;
  T* cy;
  T* uct;
  T* vct;
  T* ucx;
  T* ucy;
  T* vcx;
  T* vcy;
  T* advx;
  T* advy;
};

// C-grid quantities at x face i (y face when y = 1) of column j (row i) with
// the reference's full-array pad semantics; the inputs have materialised halos.
template <typename T>
struct FaceQ {
  T bc, vis, tang;
};

template <typename T>
__device__ FaceQ<T> face_full(const Geo<T>& g, const T* H, const T* U, const T* V, int f, int i, int j,
                              int y) {
  FaceQ<T> r{T(0.0), T(0.0), T(0.0)};
  const int m = g.m;
  const int fidx = y ? j : i;
  if (fidx < kHalo || fidx > m - kHalo) return r;
  T ph[6], pc[6], pt[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int ii = y ? i : i - kHalo + q, jj = y ? j - kHalo + q : j;
    const long o = cell(f, ii, jj, m);
    ph[q] = H[o];
    pc[q] = contra(g, o, U[o], V[o], y);
    pt[q] = y ? U[o] : V[o];
  }
  T bc = T(0.5) * (rplus(pc, 1) + rminus(pc + 1, 1));
  const int other = y ? i : j;
  const int side = y ? yface_side(j, m) : xface_side(i, m);
  if (side >= 0 && other >= kHalo && other < m - kHalo)
    bc = (bc + nb_normal_raw(g, U, V, 1, f, side, other - kHalo)) / T(2.0);
  r.bc = bc;
  r.tang = bc > T(0.0) ? rplus(pt, 1) : rminus(pt + 1, 1);
  const long o = cell(f, i, j, m);
  const T dz = y ? g.dzph_y[o] : g.dzph_x[o];
  const bool valid_mid = other >= kHalo && other <= m - kHalo;  // Poly.scalar_* core range
  const T c = celerity(valid_mid ? mid6(ph, 1) : T(0.0), dz);
  r.vis = bc + (T(4.9) / c) * (rplus(ph, 1) - rminus(ph + 1, 1));
  return r;
}

template <typename T>
__device__ T kin_full(const Geo<T>& g, const T* H, const T* U, const T* V, int f, int i, int j, int y) {
  FaceQ<T> q = face_full(g, H, U, V, f, i, j, y);
  return T(0.5) * (q.vis * q.vis + q.tang * q.tang);
}

template <typename T>
__device__ T vort_full(const Geo<T>& g, const T* H, const T* U, const T* V, int f, int i, int j) {
  const int m = g.m;
  if (i > m - 2 || j > m - 2) return T(0.0);
  const long o = cell(f, i, j, m);
  const T uy0 = face_full(g, H, U, V, f, i, j, 1).tang, uy1 = face_full(g, H, U, V, f, i, j + 1, 1).tang;
  const T vx0 = face_full(g, H, U, V, f, i, j, 0).tang, vx1 = face_full(g, H, U, V, f, i + 1, j, 0).tang;
  return g.rda[o] * (uy0 * g.d_dx[o] + vx1 * g.c_dy[o + m] - uy1 * g.d_dx[o + 1] - vx0 * g.c_dy[o]);
}

// The ten diagnostic state fields of the last stage (barotr_pure.py:158-168)
// at cell (f, i, j), over the whole padded array.
template <typename T>
__device__ void diag_cell(const Geo<T>& g, const T* H, const T* U, const T* V, const DiagOut<T>& d, int f,
                          int i, int j) {
  const int m = g.m;
  const long o = cell(f, i, j, m);
  const bool mid_ok = i >= kHalo && i <= m - kHalo && j >= kHalo && j <= m - kHalo;
  T hx = T(0.0), hy = T(0.0);
  if (mid_ok) {
    T px[6], py[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      px[q] = H[cell(f, i - kHalo + q, j, m)];
      py[q] = H[cell(f, i, j - kHalo + q, m)];
    }
    hx = mid6(px, 1);
    hy = mid6(py, 1);
  }
  d.cx[o] = celerity(hx, g.dzph_x[o]);
  d.cy[o] = celerity(hy, g.dzph_y[o]);
  const T uct = contra(g, o, U[o], V[o], 0), vct = contra(g, o, U[o], V[o], 1);
  d.uct[o] = uct;
  d.vct[o] = vct;
  const FaceQ<T> xq = face_full(g, H, U, V, f, i, j, 0);
  const FaceQ<T> yq = face_full(g, H, U, V, f, i, j, 1);
  d.ucx[o] = xq.vis;
  d.vcx[o] = xq.tang;
  d.vcy[o] = yq.vis;
  d.ucy[o] = yq.tang;
  const T vort = vort_full(g, H, U, V, f, i, j);
  if (i <= m - 2) {
    const T k0 = T(0.5) * (xq.vis * xq.vis + xq.tang * xq.tang);
    d.advx[o] = vort * vct - (kin_full(g, H, U, V, f, i + 1, j, 0) - k0) * g.rdx[o];
  } else {
    d.advx[o] = T(0.0);
  }
  if (j <= m - 2) {
    const T k0 = T(0.5) * (yq.vis * yq.vis + yq.tang * yq.tang);
    d.advy[o] = -vort * uct - (kin_full(g, H, U, V, f, i, j + 1, 1) - k0) * g.rdy[o];
  } else {
    d.advy[o] = T(0.0);
  }
}

}  // namespace bt
