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
__host__ __device__ __forceinline__ void edge_point(int side, int kk, int k, int m, int& i, int& j) {
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
// A CTA of kTileThreads threads computes one TI x TJ tile of one face.  Thread
// t works on column q = t % TJ of the tile and on the rows sl, sl + NS, ...
// (sl = t / TJ, NS = kTileThreads / TJ row slots), so a warp always covers
// consecutive columns of one row: every global access is a run of
// consecutive cells and every shared-memory stencil read is conflict-free.
//
// The stencil region of a tile is a cross: the tile's columns extended by 3
// rows on each side (the "vertical bar", read along i by the x faces) and
// the tile's rows extended by 3 columns on each side (the "horizontal bar",
// read along j by the y faces).  Each thread loads the state of its own
// interior region points straight into registers and stores the quantities
// the stencils read (h and the contravariant velocity normal to the faces
// that read the point); halo points of the region are gathered by the
// Gather items from the neighbouring face.  Constants are staged with
// cp.async in a prologue that does not depend on the state.
constexpr int kTileThreads = 256;

// Resident CTAs per SM the phase H kernels are compiled for (register cap
// 65536 / (256 * blocks)): float64 tiles need more registers per thread.  The
// float32 build with the full-tile path runs 4 (multi-wave launches: C384 7 %
// faster than at 3); the edge-path-only build, which runs the one-wave launches,
// 3 (C96 8 x 16 13.15 -> 11.93 us per substep, C48 12.43 -> 11.51).
template <typename T, bool FP = true>
struct PhaseBlocks {
  static constexpr int value = sizeof(T) == 8 ? 3 : (FP ? 4 : 3);
};
// Phase UV runs 3 CTAs per SM in both precisions: at 4 its shared-memory
// traffic throttles (MIO) and the best tile shape per size measured faster at 3.
template <typename T>
struct PhaseBlocksUV {
  static constexpr int value = 3;
};

constexpr int up4(int x) { return (x + 3) & ~3; }  // shared-memory offsets in words, 16-byte aligned

template <int TI, int TJ>
struct TileShape {
  static_assert(TJ == 16 || TJ == 32, "tile columns must be 16 or 32");
  static_assert(TI <= 32, "the east y-face column is one lane per tile row");
  static constexpr int RI = TI + 6, RJ = TJ + 6;
  static constexpr int NS = kTileThreads / TJ;      // row slots
  static constexpr int VB = RI * TJ;                // vertical-bar points (r * TJ + q)
  static constexpr int SB = 6 * TI;                 // side points: 3 W + 3 E columns per tile row
  static constexpr int NP = VB + SB;                // staged region points
  static constexpr int FX = (TI + 1) * TJ;          // x faces (a * TJ + q)
  static constexpr int FY = TI * (TJ + 1);          // y faces (r * (TJ + 1) + q)
  static constexpr int C = TI * TJ;                 // cells (a * TJ + q)
  static constexpr int EW = TI > TJ ? TI : TJ;
  // face cache block of a tile (words): the three x-face planes [3][FX], then the three y-face planes
  // [3][FY], each part padded to 16 bytes (four words)
  static constexpr int fXB = (3 * FX + 3) & ~3, fYB = (3 * FY + 3) & ~3, fW = fXB + fYB;
  static constexpr int NE = 4 * EW;                 // edge slots: 4 kinds x max(TI, TJ) positions
  static constexpr int KV = (RI + NS - 1) / NS;     // row iterations over the vertical bar
  static constexpr int KX = (TI + 1 + NS - 1) / NS; // over x-face rows
  static constexpr int KC = (TI + NS - 1) / NS;     // over tile rows
  // phase H (words): s_h [RI][RJ], s_uc [VB], s_vc [TI][RJ], s_g [NP][4], s_sn [NP],
  // s_dzx/s_cdy [FX], s_dzy/s_ddx [FY], s_rda [C], neighbour lines; s_P [FX] and
  // s_Q [FY] alias s_g (dead once the region is staged)
  static constexpr int hH = 0, hUC = up4(hH + RI * RJ), hVC = up4(hUC + VB), hG = up4(hVC + TI * RJ),
                       hSN = up4(hG + 4 * NP), hDZX = up4(hSN + NP), hCDY = up4(hDZX + FX),
                       hDZY = up4(hCDY + FX), hDDX = up4(hDZY + FY), hRDA = up4(hDDX + FY),
                       hNP = up4(hRDA + C), hNH = hNP + 6 * NE, hNDZ = hNH + 6 * NE, kWordsH = up4(hNDZ + NE);
  static constexpr int hP = hG, hQ = hG + FX;
  static_assert(FX + FY <= 4 * NP, "face fluxes must fit in the metric block they alias");
  // phase UV (words): s_v [VB], s_u [TI][RJ], s_hn [RI][RJ], s_hb [RI][RJ] (stage h of
  // the fb blend, RK3); the constants, contiguous [uG, uCEnd): cells g [C][4], sina, rda,
  // rdx, rdy, a_f, x faces c_dy, y faces d_dx; then x faces cache [3][FX], kinetic energy,
  // v_t * c_dy; y faces cache [3][FY], kinetic energy, u_t * d_dx
  static constexpr int uV = 0, uU = up4(uV + VB), uHN = up4(uU + TI * RJ), uHB = up4(uHN + RI * RJ),
                       uG = up4(uHB + RI * RJ),
                       uSN = up4(uG + 4 * C), uRDA = uSN + C, uRDX = uRDA + C, uRDY = uRDX + C, uAF = uRDY + C,
                       uCDY = up4(uAF + C), uDDX = up4(uCDY + FX), uCEnd = up4(uDDX + FY),
                       uXC = uCEnd, uKU = up4(uXC + 3 * FX), uVX = up4(uKU + FX),
                       uYC = up4(uVX + FX), uKV = up4(uYC + 3 * FY), uUY = up4(uKV + FY),
                       kWordsUV = up4(uUY + FY);
  static constexpr int uConstWords = uCEnd - uG;  // phase UV's constants of one tile
  // tile constant block (words): phase UV's constant area image, then dzph_x of the x faces [FX]
  // and dzph_y of the y faces [FY] (padded); plane offsets within the block
  static constexpr int bSN = uSN - uG, bRDA = uRDA - uG, bCDY = uCDY - uG, bDDX = uDDX - uG,
                       bDZX = uConstWords, bDZY = bDZX + FX, cW = bDZY + ((FY + 3) & ~3);
};

struct TileBox {
  int f, i0, j0, ni, nj;
};

// Work order of the tiles: the tiles on the ring of each face's tile grid
// (those touching a face edge: halo gathers and edge averages make them the
// slowest) come first, the interior tiles after them, so that the long tiles
// start in the first wave instead of finishing a launch alone (largest work
// first).  Item b < 6 R (R = ring tiles of one face) is ring tile b % R of face
// b / R; the rest are the interior tiles face by face.  Returns the tile's
// face-major, row-major index.
__device__ __forceinline__ int edge_first_tile(const Tiling& t, int b) {
  const int nti = t.nti, ntj = t.ntj;
  if (nti < 3 || ntj < 3) return b;  // every tile touches a face edge
  const int R = 2 * ntj + 2 * (nti - 2);
  int f, ti, tj;
  if (b < 6 * R) {
    f = b / R;
    int r = b - f * R;
    if (r < ntj) {
      ti = 0;
      tj = r;
    } else if ((r -= ntj) < ntj) {
      ti = nti - 1;
      tj = r;
    } else if ((r -= ntj) < nti - 2) {
      ti = 1 + r;
      tj = 0;
    } else {
      ti = 1 + r - (nti - 2);
      tj = ntj - 1;
    }
  } else {
    const int I = (nti - 2) * (ntj - 2), k = b - 6 * R;
    f = k / I;
    const int rr = k - f * I;
    ti = 1 + rr / (ntj - 2);
    tj = 1 + rr % (ntj - 2);
  }
  return (f * nti + ti) * ntj + tj;
}

// Tile number ``tile`` in face-major, row-major order.
__device__ __forceinline__ TileBox tile_box_at(const Tiling& t, int n, int tile) {
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

// The tile that work item ``item`` (a CTA of a phase launch, or a step of a
// persistent CTA's tile loop) computes, in edge_first_tile order.  The
// batched phase kernels keep the face-major order instead (tile_box_at): with
// many members in one launch the last wave is short anyway, and neighbouring
// tiles running together share their halo rows in L2 (2.7 % faster there).
__device__ __forceinline__ TileBox tile_box(const Tiling& t, int n, int item) {
  return tile_box_at(t, n, edge_first_tile(t, item));
}

// A full interior tile: TI x TJ cells whose whole stencil region (3 cells
// beyond each side) lies inside the face.  Such a tile needs no halo gather,
// no edge average and no bounds checks, so the tile phases are compiled
// separately for it (FULL = true) with its extents as constants.
__device__ __forceinline__ bool tile_full(const TileBox& b, int m, int ti, int tj) {
  return b.ni == ti && b.nj == tj && b.i0 >= 2 * kHalo && b.i0 + b.ni + kHalo <= m - kHalo &&
         b.j0 >= 2 * kHalo && b.j0 + b.nj + kHalo <= m - kHalo;
}

// 32-bit offset of cell (i, j) of face f (fields of up to 2^31 elements).
__device__ __forceinline__ int cell32(int f, int i, int j, int m) { return (f * m + i) * m + j; }

// Row handled by this thread in the tile's east y-face column (faces at column
// TJ of full-width tiles): lane r of the last warp.  With TI = 8k - 1 rows the
// x-face rows (TI + 1) fill every warp evenly and the last warp has one tile
// row fewer, so the extra column evens out the face work across the warps.
__device__ __forceinline__ int east_row() { return (int)threadIdx.x - (kTileThreads - 32); }

// Offset of a tile's face cache block (TileShape::fW words per tile, tiles in
// face-major, row-major order).  Each tile writes every face it computes into
// its own block (the faces it shares with the next tile are computed by both,
// identically), so phase UV of a tile reads only its own block: one
// contiguous range, loaded with 16-byte copies.
template <int TI, int TJ>
__device__ __forceinline__ int tile_index(const TileBox& b, int n) {
  const int nti = (n + TI - 1) / TI, ntj = (n + TJ - 1) / TJ;
  return (b.f * nti + (b.i0 - kHalo) / TI) * ntj + (b.j0 - kHalo) / TJ;
}
template <int TI, int TJ>
__device__ __forceinline__ long face_block_off(const TileBox& b, int n) {
  return (long)tile_index<TI, TJ>(b, n) * TileShape<TI, TJ>::fW;
}

// ---- asynchronous global -> shared copies ---------------------------------
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else if (BYTES == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_t(T* dst, const T* src) {
  cp_async<sizeof(T)>(dst, src);
}
template <typename T>
__device__ __forceinline__ void cp_async_mat(T* dst, const T* src) {  // 4 consecutive T
  if (sizeof(T) == 8) {
    cp_async<16>(dst, src);
    cp_async<16>(dst + 2, src + 2);
  } else {
    cp_async<16>(dst, src);
  }
}

// One 2x2 matrix (four consecutive values) or one row of it with vector
// loads: bt_plan_create and bt_round_noalloc require the matrix arrays
// (a_c2l, a_l2c, a_gct) to start on a 16-byte boundary.
__device__ __forceinline__ void ld_quad(const float* p, float* q) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  q[0] = v.x;
  q[1] = v.y;
  q[2] = v.z;
  q[3] = v.w;
}
__device__ __forceinline__ void ld_quad(const double* p, double* q) {
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  q[0] = a.x;
  q[1] = a.y;
  q[2] = b.x;
  q[3] = b.y;
}
__device__ __forceinline__ void ld_pair(const float* p, float& a, float& b) {
  const float2 v = *reinterpret_cast<const float2*>(p);
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void ld_pair(const double* p, double& a, double& b) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  a = v.x;
  b = v.y;
}

// ---- halo gathers in two steps (descriptor, then sources) ------------------
template <typename T>
struct Pull {
  int2 s;
  T w0, w1;
};
template <typename T>
__device__ __forceinline__ Pull<T> pull_desc(const Geo<T>& g, int f, int i, int j) {
  const int k = f * g.nh + halo_id(i, j, g.m);
  Pull<T> p;
  p.s = g.hsrc[k];
  p.w0 = g.hw[2 * k];
  p.w1 = g.hw[2 * k + 1];
  return p;
}

// ---- the tile's face-edge positions ----------------------------------------
// Item q of a tile's edge list: kind 0/1 = x faces of side S/N (position along
// the tile's columns), kind 2/3 = y faces of side W/E (along the tile's rows).
struct EdgeItem {
  int kind, pos, side, k;
};
// Edge positions of a tile per kind (S, N, W, E) and the routes of the
// tile's face across its four sides (8 bits each, kind order).  Scalars, not
// arrays: a dynamically indexed array would live in local memory, and each
// decode would wait on it.
struct EdgeCnt {
  int s, n, w, e, routes;
};
__device__ __forceinline__ int edge_count(const TileBox& b, int m, const int* route, EdgeCnt& c) {
  c.s = b.i0 == kHalo ? b.nj : 0;
  c.n = b.i0 + b.ni == m - kHalo ? b.nj : 0;
  c.w = b.j0 == kHalo ? b.ni : 0;
  c.e = b.j0 + b.nj == m - kHalo ? b.ni : 0;
  c.routes = route[b.f * 4 + kS] | (route[b.f * 4 + kN] << 8) | (route[b.f * 4 + kW] << 16) |
             (route[b.f * 4 + kE] << 24);
  return c.s + c.n + c.w + c.e;
}
__device__ __forceinline__ EdgeItem edge_item(const TileBox& b, const EdgeCnt& c, int q) {
  EdgeItem e;
  int kind;
  if (q < c.s) {
    kind = 0;
  } else if ((q -= c.s) < c.n) {
    kind = 1;
  } else if ((q -= c.n) < c.w) {
    kind = 2;
  } else {
    q -= c.w;
    kind = 3;
  }
  e.kind = kind;
  e.pos = q;
  e.side = kind == 0 ? kS : (kind == 1 ? kN : (kind == 2 ? kW : kE));
  e.k = kind < 2 ? (b.j0 + q - kHalo) : (b.i0 + q - kHalo);
  return e;
}

// Work items of a tile that touches face edges, spread over the whole CTA:
//   item t < 3P:  halo point at depth t % 3 outside edge position t / 3 of the
//                 tile: its h and normal contravariant velocity (phase H), or
//                 its raw tangential-reading velocity and new h (phase UV) --
//                 read directly when the stored halo is valid, else gathered
//                 from the neighbouring face;
//   item t >= 3P: point q = (t - 3P) % 6 of the neighbour's 6-point line normal
//                 to the shared edge at position (t - 3P) / 6: its contravariant
//                 normal velocity (and h for the mass-flux average).
// P is the number of edge positions of the tile.  Descriptor loads of all
// items go out in a first sweep, source loads in a second, so a CTA waits for
// two L2 round trips instead of one chain per point.
struct ItemCell {
  int f, i, j;      // cell whose value the item needs
  int o;            // its offset within the member, cell32(f, i, j, m)
  int kind;         // edge kind 0..3 (S, N, W, E)
  int r, c;         // region row / column (region items)
  int slot;         // line item: edge slot * 6 + q
  int line, y, q;   // line item: 1, normal axis (1 = y), point index
};

// Shared-memory words (ints) past a phase's layout where each thread keeps
// its first gather item, decoded in the prologue: the offset o at [t] and the
// other fields the item needs at [kTileThreads + t], packed as
// r | c << 6 | slot << 12 | line << 22 | kind << 23 | y << 25 | (q == 3) << 26.
// Only the writing thread reads them back (after the grid dependency), so the
// decode's cold code stays off the critical path without holding registers.
constexpr int kItemWords = 2 * kTileThreads;
__device__ __forceinline__ int pack_item(const ItemCell& c) {
  return c.r | (c.c << 6) | (c.slot << 12) | (c.line << 22) | (c.kind << 23) | (c.y << 25) | ((c.q == 3) << 26);
}
__device__ __forceinline__ ItemCell unpack_item(int o, int pk) {
  ItemCell c;
  c.f = c.i = c.j = 0;  // not needed past the descriptor sweep
  c.o = o;
  c.r = pk & 63;
  c.c = (pk >> 6) & 63;
  c.slot = (pk >> 12) & 1023;
  c.line = (pk >> 22) & 1;
  c.kind = (pk >> 23) & 3;
  c.y = (pk >> 25) & 1;
  c.q = ((pk >> 26) & 1) ? 3 : 0;
  return c;
}

__device__ __forceinline__ ItemCell decode_item(const TileBox& b, const EdgeCnt& cnt, int P, int t, int m, int n,
                                                int EW) {
  ItemCell c;
  if (t < 3 * P) {
    const EdgeItem e = edge_item(b, cnt, t / 3);
    const int d = t % 3;
    int r, cc;
    switch (e.kind) {
      case 0: r = d; cc = e.pos + kHalo; break;                  // S: region rows 0..2
      case 1: r = b.ni + kHalo + d; cc = e.pos + kHalo; break;   // N: rows ni+3..ni+5
      case 2: r = e.pos + kHalo; cc = d; break;                  // W: region cols 0..2
      default: r = e.pos + kHalo; cc = b.nj + kHalo + d; break;  // E: cols nj+3..nj+5
    }
    c.f = b.f;
    c.i = b.i0 - kHalo + r;
    c.j = b.j0 - kHalo + cc;
    c.o = cell32(c.f, c.i, c.j, m);
    c.kind = e.kind;
    c.r = r;
    c.c = cc;
    c.slot = 0;
    c.line = 0;
    c.y = 0;
    c.q = 0;
  } else {
    const int t2 = t - 3 * P;
    const EdgeItem e = edge_item(b, cnt, t2 / 6);
    const int q = t2 % 6;
    const int r = (cnt.routes >> (8 * e.kind)) & 0xff;
    const int ns = route_side(r);
    const int kk = route_rev(r) ? n - 1 - e.k : e.k;
    c.f = route_nb(r);
    edge_point(ns, kk, q, m, c.i, c.j);
    c.o = cell32(c.f, c.i, c.j, m);
    c.kind = e.kind;
    c.r = 0;
    c.c = 0;
    c.slot = (e.kind * EW + e.pos) * 6 + q;
    c.line = 1;
    c.y = (ns == kE || ns == kW);
    c.q = q;
  }
  return c;
}

// Shared-memory destinations of the gather items of one phase.
template <typename T>
struct GatherSink {
  T* h;    // H: region h [RI][RJ]        UV: blended new h [RI][RJ]
  T* vb;   // H: s_uc [VB]                UV: raw v [VB]
  T* hb;   // H: s_vc [TI][RJ]            UV: raw u [TI][RJ]
  T* np;   // H: neighbour lines (contravariant normal velocity, h, depth)
  T* nh;
  T* ndz;
  // tile-resident round only (RES): phase H also leaves the raw velocities of
  // the region halo in phase UV's arrays, and phase UV blends with the stage
  // h phase H staged
  T* rv = nullptr;        // H: phase UV's raw v [VB]
  T* ru = nullptr;        // H: phase UV's raw u [TI][RJ]
  const T* hs = nullptr;  // UV: phase H's region h [RI][RJ]
};

// Shared-memory pointers of the tile-resident round kernel: phase H and phase
// UV keep separate layouts, so constants and the face cache stay in place
// for the whole round.
template <typename T>
struct ResSm {
  T* uv;      // phase UV layout (constants, face cache, raw velocities of the stage)
  T* pq;      // phase H face fluxes [FX + FY] (alias the metric block otherwise)
  T* hs;      // phase H region h [RI][RJ]: the stage h of the fb blend in phase UV
  int* items; // gather item scratch (kItemWords)
};

template <typename T, int TI, int TJ, bool UV, bool RES = false>
struct Gather {
  using S = TileShape<TI, TJ>;
  // phase H gathers the region halo and the neighbour edge lines (9 items per
  // edge position); phase UV only the region halo (3 per position)
  static constexpr int kPerPos = UV ? 3 : 9;
  Pull<T> pd;  // descriptor of the thread's first item
  bool pl;

  __device__ __forceinline__ static bool needs_pull(const StageIO<T>& io, const ItemCell& c, int m) {
    return !is_interior(c.i, c.j, m) && (!io.stored_halo || (UV && !c.line));
  }

  // sweep 1: the descriptor of the thread's first item (constants, may
  // precede the grid dependency)
  __device__ __forceinline__ void descriptors(const Geo<T>& g, const StageIO<T>& io, const TileBox& b,
                                              const EdgeCnt& cnt, int P, int* s_items) {
    pl = false;
    pd.s = make_int2(0, 0);
    pd.w0 = pd.w1 = T(0.0);
    if ((int)threadIdx.x < kPerPos * P) {
      const ItemCell c = decode_item(b, cnt, P, threadIdx.x, g.m, g.n, S::EW);
      s_items[threadIdx.x] = c.o;
      s_items[kTileThreads + threadIdx.x] = pack_item(c);
      if (needs_pull(io, c, g.m)) {
        pd = pull_desc(g, c.f, c.i, c.j);
        pl = true;
      }
    }
  }

  // One item.  Every lane issues the same loads whatever its item's kind --
  // the two sources of an interpolated halo value, or the cell itself twice
  // for a direct read -- so a warp mixing kinds waits for one memory round
  // trip, not one per kind; the results are selected afterwards (a direct
  // read stays exact), and all loads precede the item's shared-memory stores.
  __device__ __forceinline__ void one(const Geo<T>& g, const StageIO<T>& io, const ItemCell& c, const Pull<T>& p,
                                      bool pull, const GatherSink<T>& k) {
    if constexpr (UV && RES) {
      // resident phase UV: the raw velocities and the stage h of the halo
      // point were staged by phase H; only the new h is interpolated here
      T hn = p.w0 * ((const T*)io.h_out)[p.s.x] + p.w1 * ((const T*)io.h_out)[p.s.y];
      const int e = c.r * S::RJ + c.c;
      if (io.beta != T(0.0)) hn = (T(1.0) - io.beta) * hn + io.beta * k.hs[e];  // fb_scheme
      k.h[e] = hn;
      return;
    }
    const int o = c.o;
    const bool vpull = UV ? !io.stored_halo : pull;  // velocity interpolated (else read directly)
    const int sa = vpull ? p.s.x : o, sb = vpull ? p.s.y : o;
    const T ua = io.u[sa], va = io.v[sa], ub = io.u[sb], vb = io.v[sb];
    T c0[4], c1[4], l2[4];
    ld_quad(g.c2l + 4 * (long)sa, c0);
    ld_quad(g.c2l + 4 * (long)sb, c1);
    ld_quad(g.l2c + 4 * (long)o, l2);
    if (!UV) {
      const bool want_h = !c.line || io.last;  // region h, or the neighbour h of the mass-flux average
      T ha = T(0.0), hb = T(0.0), dz = T(0.0);
      if (want_h) {
        ha = io.h[sa];
        hb = io.h[sb];
      }
      const bool yaxis = c.line ? c.y : c.kind >= 2;  // contravariant component normal to the faces read
      T g0, g1;
      ld_pair(g.gct + 4 * (long)o + (yaxis ? 2 : 0), g0, g1);
      const T sn = g.sina[o];
      if (c.line && want_h && c.q == 3) dz = (c.y ? g.dzph_y : g.dzph_x)[o];
      T u = ua, v = va, h = ha;
      if (vpull) {  // ext_vector / ext_scalar, cube.py:130-153
        const T ull0 = c0[0] * ua + c0[1] * va, vll0 = c0[2] * ua + c0[3] * va;
        const T ull1 = c1[0] * ub + c1[1] * vb, vll1 = c1[2] * ub + c1[3] * vb;
        const T ull = p.w0 * ull0 + p.w1 * ull1;
        const T vll = p.w0 * vll0 + p.w1 * vll1;
        u = l2[0] * ull + l2[1] * vll;
        v = l2[2] * ull + l2[3] * vll;
        h = p.w0 * ha + p.w1 * hb;
      }
      const T ct = (g0 * u + g1 * v) * sn;  // remap.py:34-39
      if (!c.line) {
        k.h[c.r * S::RJ + c.c] = h;
        if (c.kind < 2)  // S/N halo rows belong to the vertical bar
          k.vb[c.r * TJ + (c.c - kHalo)] = ct;
        else
          k.hb[(c.r - kHalo) * S::RJ + c.c] = ct;
        if constexpr (RES) {  // phase UV's raw (tangential-reading) velocity at the same point
          if (c.kind < 2)
            k.rv[c.r * TJ + (c.c - kHalo)] = v;
          else
            k.ru[(c.r - kHalo) * S::RJ + c.c] = u;
        }
      } else {
        k.np[c.slot] = ct;
        if (want_h) {
          k.nh[c.slot] = h;
          if (c.q == 3) k.ndz[c.slot / 6] = dz;
        }
      }
    } else {  // region items only; the new h never has a stored halo
      const bool blend = io.beta != T(0.0);
      const T n0 = ((const T*)io.h_out)[p.s.x], n1 = ((const T*)io.h_out)[p.s.y];
      T ba = T(0.0), bb = T(0.0);
      if (blend) {
        ba = io.h[sa];
        bb = io.h[sb];
      }
      T u = ua, v = va, h = ba;
      if (vpull) {
        const T ull0 = c0[0] * ua + c0[1] * va, vll0 = c0[2] * ua + c0[3] * va;
        const T ull1 = c1[0] * ub + c1[1] * vb, vll1 = c1[2] * ub + c1[3] * vb;
        const T ull = p.w0 * ull0 + p.w1 * ull1;
        const T vll = p.w0 * vll0 + p.w1 * vll1;
        u = l2[0] * ull + l2[1] * vll;
        v = l2[2] * ull + l2[3] * vll;
        h = p.w0 * ba + p.w1 * bb;
      }
      T hn = p.w0 * n0 + p.w1 * n1;
      if (blend) hn = (T(1.0) - io.beta) * hn + io.beta * h;  // fb_scheme, barotr_pure.py:52-54
      k.h[c.r * S::RJ + c.c] = hn;
      if (c.kind < 2)
        k.vb[c.r * TJ + (c.c - kHalo)] = v;
      else
        k.hb[(c.r - kHalo) * S::RJ + c.c] = u;
    }
  }

  // sweep 2: sources (state, after the grid dependency) and the items'
  // values.  One rolled loop, so the item code exists once in the kernel (the
  // edge path is cold code: at small sizes each CTA runs it once and waits on
  // instruction fetch); items past the first of a thread (tiles with more than
  // kTileThreads items) load their descriptor here.
  __device__ __forceinline__ void sources(const Geo<T>& g, const StageIO<T>& io, const TileBox& b,
                                          const EdgeCnt& cnt, int P, const GatherSink<T>& k, const int* s_items) {
    const int nitems = kPerPos * P;
#pragma unroll 1
    for (int t = threadIdx.x; t < nitems; t += kTileThreads) {
      bool pull = pl;
      Pull<T> p = pd;
      ItemCell c;
      if (t < kTileThreads) {
        c = unpack_item(s_items[t], s_items[kTileThreads + t]);
      } else {
        c = decode_item(b, cnt, P, t, g.m, g.n, S::EW);
        pull = needs_pull(io, c, g.m);
        if (pull) p = pull_desc(g, c.f, c.i, c.j);
      }
      one(g, io, c, p, pull, k);
    }
  }
};

// Normal velocity of the neighbour's line (6 contravariant values) before averaging.
template <typename T>
__device__ __forceinline__ T line_raw(const T* np) {
  return T(0.5) * (rplus(np, 1) + rminus(np + 1, 1));
}

// Wait for the previous kernel of the stream (programmatic dependent launch);
// a no-op when the kernel was launched without a programmatic dependency.
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
// Allow the next kernel of the stream to start its prologue.
__device__ __forceinline__ void release_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// Celerity sqrt(g (h + dz)) with the 10 m/s floor and the viscosity
// coefficient 4.9 / celerity (barotr_pure.py:21-33).  float64 keeps IEEE
// sqrt and division like the reference; the float32 form takes the
// reciprocal square root once (sqrt = x * rsqrt(x)), with the same floor and
// NaN propagation.
template <typename T>
__device__ __forceinline__ void celerity_coef(T hface, T dz, T& c, T& coef) {
  if constexpr (sizeof(T) == 8) {
    c = celerity(hface, dz);
    coef = T(4.9) / c;
  } else {
    const float x = 9.8f * (hface + dz);
    if (x > 0.0f) {
      const float r = rsqrtf(x);
      c = x * r;
      coef = 4.9f * r;
      if (c < 10.0f) {
        c = 10.0f;
        coef = 0.49f;
      }
    } else {  // zero, negative depth or NaN: the exact path
      c = celerity(hface, dz);
      coef = 4.9f / c;
    }
  }
}

// Region points a thread stages itself: interior points, and halo points that
// no gather item covers -- the halo rows (columns) that the region of a tile
// next to a tile thinner than 3 cells reaches without the tile touching that
// face edge; those are fetched point by point.
struct EdgeCover {
  bool s, n, w, e;  // the tile touches face edge S / N / W / E (its halo points there are gather items)
  __device__ __forceinline__ EdgeCover(const TileBox& b, int m)
      : s(b.i0 == kHalo), n(b.i0 + b.ni == m - kHalo), w(b.j0 == kHalo), e(b.j0 + b.nj == m - kHalo) {}
  __device__ __forceinline__ bool row_staged(int i, int m) const {
    return !((i < kHalo && s) || (i >= m - kHalo && n));
  }
  __device__ __forceinline__ bool col_staged(int j, int m) const {
    return !((j < kHalo && w) || (j >= m - kHalo && e));
  }
};

// ---- phase H ----------------------------------------------------------------
template <typename T, int TI, int TJ>
struct LayoutH {
  using S = TileShape<TI, TJ>;
  T *s_h, *s_uc, *s_vc, *s_g, *s_sn, *s_dzx, *s_cdy, *s_dzy, *s_ddx, *s_rda, *s_P, *s_Q, *s_np, *s_nh, *s_ndz;
  __device__ __forceinline__ explicit LayoutH(T* sm) {
    s_h = sm + S::hH;
    s_uc = sm + S::hUC;
    s_vc = sm + S::hVC;
    s_g = sm + S::hG;
    s_sn = sm + S::hSN;
    s_dzx = sm + S::hDZX;
    s_cdy = sm + S::hCDY;
    s_dzy = sm + S::hDZY;
    s_ddx = sm + S::hDDX;
    s_rda = sm + S::hRDA;
    s_P = sm + S::hP;
    s_Q = sm + S::hQ;
    s_np = sm + S::hNP;
    s_nh = sm + S::hNH;
    s_ndz = sm + S::hNDZ;
  }
};

template <typename T, int TI, int TJ>
struct LayoutUV {
  using S = TileShape<TI, TJ>;
  T *s_v, *s_u, *s_hn, *s_hb, *s_g, *s_sn, *s_rda, *s_rdx, *s_rdy, *s_af, *s_xc, *s_cdy, *s_ku, *s_vx, *s_yc,
      *s_ddx, *s_kv, *s_uy;
  __device__ __forceinline__ explicit LayoutUV(T* sm) {
    s_v = sm + S::uV;
    s_u = sm + S::uU;
    s_hn = sm + S::uHN;
    s_hb = sm + S::uHB;
    s_g = sm + S::uG;
    s_sn = sm + S::uSN;
    s_rda = sm + S::uRDA;
    s_rdx = sm + S::uRDX;
    s_rdy = sm + S::uRDY;
    s_af = sm + S::uAF;
    s_xc = sm + S::uXC;
    s_cdy = sm + S::uCDY;
    s_ku = sm + S::uKU;
    s_vx = sm + S::uVX;
    s_yc = sm + S::uYC;
    s_ddx = sm + S::uDDX;
    s_kv = sm + S::uKV;
    s_uy = sm + S::uUY;
  }
};

// 16-byte copies of ``words`` words (a multiple of 16 bytes) from global src to shared dst.
template <typename T, int WORDS>
__device__ __forceinline__ void cp_async_run(T* dst, const T* src) {
  constexpr int V = 16 / sizeof(T);
  static_assert(WORDS % V == 0, "runs of whole 16-byte chunks");
#pragma unroll
  for (int w = threadIdx.x * V; w < WORDS; w += kTileThreads * V) cp_async<16>(dst + w, src + w);
}

// Phase H constants of a full interior tile from the tile constant blocks: the
// region metric (vertical bar: 3 rows of the tile above, the tile's own rows, 3
// rows of the tile below; side points: 3 columns of the tiles left and right --
// all four exist on the same face for a full tile and hold at least 3 rows /
// columns) and the tile's own face and cell constants, in 16-byte copies.
template <typename T, int TI, int TJ>
__device__ __forceinline__ void tile_h_consts_blocks(const Geo<T>& g, const TileBox& b, T* sm) {
  using S = TileShape<TI, TJ>;
  const LayoutH<T, TI, TJ> L(sm);
  const int ntj = (g.n + TJ - 1) / TJ;
  const T* own = g.cblk + (long)tile_index<TI, TJ>(b, g.n) * S::cW;
  const T* above = own - (long)ntj * S::cW;
  const T* below = own + (long)ntj * S::cW;
  const T* left = own - S::cW;
  const T* right = own + S::cW;
  cp_async_run<T, 4 * 3 * TJ>(L.s_g, above + 4 * (TI - 3) * TJ);
  cp_async_run<T, 4 * TI * TJ>(L.s_g + 4 * 3 * TJ, own);
  cp_async_run<T, 4 * 3 * TJ>(L.s_g + 4 * (TI + 3) * TJ, below);
  cp_async_run<T, 3 * TJ>(L.s_sn, above + S::bSN + (TI - 3) * TJ);
  cp_async_run<T, TI * TJ>(L.s_sn + 3 * TJ, own + S::bSN);
  cp_async_run<T, 3 * TJ>(L.s_sn + (TI + 3) * TJ, below + S::bSN);
  if (threadIdx.x < 6 * TI) {  // side point (r, c): columns TJ-3.. of the left tile, 0..2 of the right one
    const int t = threadIdx.x, r = t / 6, c = t - 6 * r;
    const T* nb = c < 3 ? left : right;
    const int e = c < 3 ? r * TJ + TJ - 3 + c : r * TJ + c - 3;  // the cell within the neighbour's block
    cp_async_mat(L.s_g + 4 * (S::VB + t), nb + 4 * e);            // metric plane first, 4 words per cell
    cp_async_t(L.s_sn + S::VB + t, nb + S::bSN + e);
  }
  cp_async_run<T, S::C>(L.s_rda, own + S::bRDA);
  cp_async_run<T, S::FX>(L.s_cdy, own + S::bCDY);
  cp_async_run<T, S::FX>(L.s_dzx, own + S::bDZX);
  cp_async_run<T, (S::FY + 3) & ~3>(L.s_ddx, own + S::bDDX);
  cp_async_run<T, (S::FY + 3) & ~3>(L.s_dzy, own + S::bDZY);
}

// Phase H constants of the tile (cp.async, not yet awaited).
template <typename T, int TI, int TJ, bool FULL>
__device__ __forceinline__ void tile_h_consts(const Geo<T>& g, const TileBox& b, T* sm) {
  using S = TileShape<TI, TJ>;
  if (FULL && g.cblk != nullptr && g.cblk_ti == TI && g.cblk_tj == TJ) {
    tile_h_consts_blocks<T, TI, TJ>(g, b, sm);
    return;
  }
  const LayoutH<T, TI, TJ> L(sm);
  const int m = g.m, q = threadIdx.x % TJ, sl = threadIdx.x / TJ;
  const int ni = FULL ? TI : b.ni, nj = FULL ? TJ : b.nj;
  // region metric (halo points of edge tiles are also read by the gather items, from global memory)
  if (q < nj) {
    const int o0 = cell32(b.f, b.i0 - kHalo, b.j0 + q, m);
#pragma unroll
    for (int k = 0; k < S::KV; ++k) {
      const int r = sl + k * S::NS;
      if (r < ni + 6) {
        const int o = o0 + r * m, p = r * TJ + q;
        cp_async_mat(L.s_g + 4 * p, g.gct + 4 * (long)o);
        cp_async_t(L.s_sn + p, g.sina + o);
      }
    }
  }
  if (threadIdx.x < 6 * ni) {
    const int t = threadIdx.x, r = t / 6, c = t - 6 * r, cc = c < 3 ? c : nj + c;
    const int o = cell32(b.f, b.i0 + r, b.j0 - kHalo + cc, m), p = S::VB + t;
    cp_async_mat(L.s_g + 4 * p, g.gct + 4 * (long)o);
    cp_async_t(L.s_sn + p, g.sina + o);
  }
  // face and cell constants
  if (q < nj) {
    const int o0 = cell32(b.f, b.i0, b.j0 + q, m);
#pragma unroll
    for (int k = 0; k < S::KX; ++k) {
      const int a = sl + k * S::NS;
      if (a <= ni) {
        cp_async_t(L.s_dzx + a * TJ + q, g.dzph_x + o0 + a * m);
        cp_async_t(L.s_cdy + a * TJ + q, g.c_dy + o0 + a * m);
      }
    }
#pragma unroll
    for (int k = 0; k < S::KC; ++k) {
      const int a = sl + k * S::NS;
      if (a < ni) cp_async_t(L.s_rda + a * TJ + q, g.rda + o0 + a * m);
    }
  }
  if (q <= nj) {
    const int o0 = cell32(b.f, b.i0, b.j0 + q, m);
#pragma unroll
    for (int k = 0; k < S::KC; ++k) {
      const int r = sl + k * S::NS;
      if (r < ni) {
        cp_async_t(L.s_dzy + r * (TJ + 1) + q, g.dzph_y + o0 + r * m);
        cp_async_t(L.s_ddx + r * (TJ + 1) + q, g.d_dx + o0 + r * m);
      }
    }
  }
  if (nj == TJ && east_row() >= 0 && east_row() < ni) {  // the last y-face column of full-width tiles
    const int r = east_row(), o = cell32(b.f, b.i0 + r, b.j0 + TJ, m);
    cp_async_t(L.s_dzy + r * (TJ + 1) + TJ, g.dzph_y + o);
    cp_async_t(L.s_ddx + r * (TJ + 1) + TJ, g.d_dx + o);
  }
}

// Halo-gather descriptors of a tile phase (edge tiles; P = 0 for full tiles).
template <typename T, int TI, int TJ, bool FULL, bool UV, bool RES>
__device__ __forceinline__ void tile_desc(const Geo<T>& g, const StageIO<T>& io, const TileBox& b,
                                          Gather<T, TI, TJ, UV, RES>& gat, EdgeCnt& cnt, int& P, int* items) {
  if (FULL) {
    P = 0;
  } else {
    P = edge_count(b, g.m, g.route, cnt);
    if (P > 0) gat.descriptors(g, io, b, cnt, P, items);
  }
}

// Phase H prologue: constants of the tile (cp.async, not yet awaited) and the
// halo-gather descriptors.  Independent of the state, so it may run before the
// previous phase has finished (programmatic launch, or before a grid barrier).
template <typename T, int TI, int TJ, bool FULL>
__device__ __forceinline__ void tile_h_pro_t(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                             Gather<T, TI, TJ, false>& gat, EdgeCnt& cnt, int& P) {
  using S = TileShape<TI, TJ>;
  tile_h_consts<T, TI, TJ, FULL>(g, b, sm);
  tile_desc<T, TI, TJ, FULL, false, false>(g, io, b, gat, cnt, P, reinterpret_cast<int*>(sm + S::kWordsH));
}

// The neighbour's side of every edge face of a tile, from its gathered 6-point
// lines (slot = edge kind x EW + position): its raw C-grid normal velocity
// (line_raw) replaces the line's first velocity value and, on the last stage,
// its reconstructed face h values and celerity viscosity coefficient replace
// the line's first three h values.  Run between the staging barriers, one edge
// position per thread counted from the CTA's last thread (the threads with the
// fewest region points), so that the face pass of an edge face carries one
// square root and division chain instead of two.  float64 only: measured on a
// B200 it shortens the float64 round (C96 16.60 -> 16.15 us per substep, C384
// 160.3 -> 157.9) and lengthens the float32 one (C384 69.1 -> 70.7, C768
// 293.5 -> 313.4), whose face chains are short and whose extra staging pass
// costs more than it saves.
template <typename T>
__host__ __device__ constexpr bool edge_lines_staged() { return sizeof(T) == 8; }

template <typename T, int EW>
__device__ __forceinline__ void edge_lines(const StageIO<T>& io, const TileBox& b, const EdgeCnt& cnt, int P, T* s_np,
                                           T* s_nh, const T* s_ndz) {
  for (int k = kTileThreads - 1 - (int)threadIdx.x; k < P; k += kTileThreads) {
    const EdgeItem e = edge_item(b, cnt, k);
    const int slot = e.kind * EW + e.pos;
    T* np = s_np + 6 * slot;
    const T lr = line_raw(np);
    if (io.last) {
      T* nh = s_nh + 6 * slot;
      const T nhe = rplus(nh, 1), nhw = rminus(nh + 1, 1);
      T nc, ncoef;
      celerity_coef(mid6(nh, 1), s_ndz[slot], nc, ncoef);
      nh[0] = nhe;
      nh[1] = nhw;
      nh[2] = ncoef;
    }
    np[0] = lr;
  }
}

// Phase H of one x face or y face: C-grid normal velocity (remap.py:41-55)
// and its edge average (communication.py:504-570), upwind mass flux with the
// celerity-based velocity viscosity (barotr_pure.py:21-49) and its edge
// average on the last stage, and the face cache of phase UV.
// ph / pu: the 6 h / contravariant values along the face normal (strides sh / su).
template <typename T>
__device__ __forceinline__ T face_h(const StageIO<T>& io, const T* ph, int sh, const T* pu, int su, int side,
                                    int slot, T dz, const T* s_np, const T* s_nh, const T* s_ndz, T* fc,
                                    int pstride) {
  T hh[6], uu[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    hh[k] = ph[k * sh];
    uu[k] = pu[k * su];
  }
  const T ue = rplus(uu, 1), uw = rminus(uu + 1, 1);
  T bc = T(0.5) * (ue + uw);
  if (side >= 0) {  // the neighbour's raw normal velocity
    const T nraw = edge_lines_staged<T>() ? s_np[6 * slot] : line_raw(s_np + 6 * slot);
    bc = (bc + nraw) / T(2.0);
  }
  const T he = rplus(hh, 1), hw = rminus(hh + 1, 1);
  T cc, coef;
  celerity_coef(mid6(hh, 1), dz, cc, coef);
  const T vis = bc + coef * (he - hw);
  T fl = dz * vis + (vis > T(0.0) ? he : hw) * vis;
  if (io.last && side >= 0) {  // the neighbour's flux at the same edge face (barotr_pure.py:29-49)
    const T* nh = s_nh + 6 * slot;
    const T ndz = s_ndz[slot];
    T nhe, nhw, ncoef;
    if constexpr (edge_lines_staged<T>()) {  // its face values and viscosity coefficient, staged
      nhe = nh[0];
      nhw = nh[1];
      ncoef = nh[2];
    } else {
      nhe = rplus(nh, 1);
      nhw = rminus(nh + 1, 1);
      T nc;
      celerity_coef(mid6(nh, 1), ndz, nc, ncoef);
    }
    const T nvis = bc + ncoef * (nhe - nhw);
    fl = (fl + (ndz * nvis + (nvis > T(0.0) ? nhe : nhw) * nvis)) / T(2.0);
  }
  // face cache for phase UV: three planes pstride apart
  fc[0] = bc;
  fc[pstride] = vis;
  fc[2 * pstride] = T(0.5) * cc * (ue - uw);  // celerity viscosity flux, barotr_pure.py:68-69
  return fl;
}

// Phase H of one tile: writes the new h on the tile's interior cells.
// RES (tile-resident round): the constants are already in shared memory, the
// face fluxes get their own area, and the face cache and the raw velocities
// of the region go to phase UV's layout (rs.uv) instead of global memory.
template <typename T, int TI, int TJ, bool FULL, bool RES = false>
__device__ __forceinline__ void tile_h_main_t(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                              Gather<T, TI, TJ, false, RES>& gat, const EdgeCnt& cnt, int P,
                                              const ResSm<T>& rs = ResSm<T>{}) {
  using S = TileShape<TI, TJ>;
  constexpr int RJ = S::RJ;
  static_assert(6 * TI <= kTileThreads, "one side point per thread");
  const int m = g.m, n = g.n, f = b.f, q = threadIdx.x % TJ, sl = threadIdx.x / TJ;
  const int ni = FULL ? TI : b.ni, nj = FULL ? TJ : b.nj;
  LayoutH<T, TI, TJ> L(sm);
  const LayoutUV<T, TI, TJ> U(RES ? rs.uv : sm);  // RES only
  if constexpr (RES) {
    L.s_P = rs.pq;
    L.s_Q = rs.pq + S::FX;
  }
  int* const items = RES ? rs.items : reinterpret_cast<int*>(sm + S::kWordsH);
  // state of the thread's interior region points and base h of its cells, into registers
  T hv[S::KV], uv[S::KV], vv[S::KV], hpc[S::KC];
  T hs = T(0.0), us = T(0.0), vs = T(0.0);
  const EdgeCover ec(b, m);
  const int ov = cell32(f, b.i0 - kHalo, b.j0 + q, m);
#pragma unroll
  for (int k = 0; k < S::KV; ++k) {
    const int r = sl + k * S::NS, i = b.i0 - kHalo + r;
    if (q < nj && r < ni + 6 && (FULL || (i >= kHalo && i < m - kHalo))) {  // halo rows: see below
      const int o = ov + r * m;
      hv[k] = io.h[o];
      uv[k] = io.u[o];
      vv[k] = io.v[o];
    }
  }
  const int t6 = threadIdx.x;
  const int sr = t6 / 6, sc = t6 - 6 * sr, scc = sc < 3 ? sc : nj + sc, sj = b.j0 - kHalo + scc;
  const bool side_pt = t6 < 6 * ni && (FULL || ec.col_staged(sj, m));
  if (side_pt) {
    if (FULL || (sj >= kHalo && sj < m - kHalo)) {
      const int o = cell32(f, b.i0 + sr, sj, m);
      hs = io.h[o];
      us = io.u[o];
      vs = io.v[o];
    } else {
      hs = fetch_s(io.h, g, f, b.i0 + sr, sj, io.stored_halo);
      fetch_v(io.u, io.v, g, f, b.i0 + sr, sj, io.stored_halo, us, vs);
    }
  }
#pragma unroll
  for (int k = 0; k < S::KC; ++k) {
    const int a = sl + k * S::NS;
    if (q < nj && a < ni) hpc[k] = io.hp[ov + (a + kHalo) * m];
  }
  if (!FULL && P > 0) {
    GatherSink<T> sink{L.s_h, L.s_uc, L.s_vc, L.s_np, L.s_nh, L.s_ndz};
    if constexpr (RES) {
      sink.rv = U.s_v;
      sink.ru = U.s_u;
    }
    gat.sources(g, io, b, cnt, P, sink, items);
  }
  cp_async_wait_all();
  __syncthreads();

  // h and contravariant velocities of the region (remap.py:34-39)
#pragma unroll
  for (int k = 0; k < S::KV; ++k) {
    const int r = sl + k * S::NS, i = b.i0 - kHalo + r;
    if (q < nj && r < ni + 6 && (FULL || (i >= kHalo && i < m - kHalo))) {
      const int p = r * TJ + q;
      const T* G = L.s_g + 4 * p;
      const T sn = L.s_sn[p], u = uv[k], v = vv[k];
      const bool row = r >= kHalo && r < ni + kHalo;
      L.s_h[r * RJ + q + kHalo] = hv[k];
      L.s_uc[p] = (G[0] * u + G[1] * v) * sn;
      if (row) L.s_vc[(r - kHalo) * RJ + q + kHalo] = (G[2] * u + G[3] * v) * sn;
      if constexpr (RES) {  // phase UV's raw velocities (tangential reconstructions)
        U.s_v[p] = v;
        if (row) U.s_u[(r - kHalo) * RJ + q + kHalo] = u;
      }
    }
  }
  if (!FULL) {
    // halo rows of the region that no gather item covers (EdgeCover), fetched
    // point by point; a rolled loop keeps this rarely run code small
#pragma unroll 1
    for (int k = 0; k < S::KV; ++k) {
      const int r = sl + k * S::NS, i = b.i0 - kHalo + r;
      if (q < nj && r < ni + 6 && ec.row_staged(i, m) && !(i >= kHalo && i < m - kHalo)) {
        T u, v;
        const T h = fetch_s(io.h, g, f, i, b.j0 + q, io.stored_halo);
        fetch_v(io.u, io.v, g, f, i, b.j0 + q, io.stored_halo, u, v);
        const int p = r * TJ + q;
        const T* G = L.s_g + 4 * p;
        const T sn = L.s_sn[p];
        L.s_h[r * RJ + q + kHalo] = h;
        L.s_uc[p] = (G[0] * u + G[1] * v) * sn;
        if constexpr (RES) U.s_v[p] = v;
      }
    }
  }
  if (side_pt) {
    const T* G = L.s_g + 4 * (S::VB + t6);
    const T sn = L.s_sn[S::VB + t6];
    L.s_h[(sr + kHalo) * RJ + scc] = hs;
    L.s_vc[sr * RJ + scc] = (G[2] * us + G[3] * vs) * sn;
    if constexpr (RES) U.s_u[sr * RJ + scc] = us;
  }
  if (edge_lines_staged<T>() && !FULL && P > 0) edge_lines<T, S::EW>(io, b, cnt, P, L.s_np, L.s_nh, L.s_ndz);
  __syncthreads();

  // faces; their fluxes (times c_dy / d_dx) alias the metric block, no longer read.  The face
  // cache of every face goes to the tile's block (phase UV's shared-memory layout when resident)
  T* const fblk = RES ? nullptr : io.fx + face_block_off<TI, TJ>(b, n);
  if (q < nj) {
#pragma unroll
    for (int k = 0; k < S::KX; ++k) {
      const int a = sl + k * S::NS;
      if (a <= ni) {
        const int side =
            FULL ? -1 : ((a == 0 && b.i0 == kHalo) ? kS : ((a == ni && b.i0 + ni == m - kHalo) ? kN : -1));
        const int e = a * TJ + q;
        T* fc = RES ? U.s_xc + e : fblk + e;
        const T fl = face_h<T>(io, L.s_h + a * RJ + q + kHalo, RJ, L.s_uc + a * TJ + q, TJ, side,
                               (side == kS ? 0 : 1) * S::EW + q, L.s_dzx[e], L.s_np, L.s_nh, L.s_ndz, fc, S::FX);
        L.s_P[e] = fl * L.s_cdy[e];
      }
    }
  }
  // y faces: (r, qq) with qq = q, plus qq = TJ for full-width tiles (lanes of the last warp)
#pragma unroll
  for (int k = 0; k <= S::KC; ++k) {
    int r, qq;
    if (k < S::KC) {
      r = sl + k * S::NS;
      qq = q;
      if (r >= ni || q > nj) continue;
    } else {
      r = east_row();
      qq = TJ;
      if (nj != TJ || r < 0 || r >= ni) continue;
    }
    const int side =
        FULL ? -1 : ((qq == 0 && b.j0 == kHalo) ? kW : ((qq == nj && b.j0 + nj == m - kHalo) ? kE : -1));
    const int e = r * (TJ + 1) + qq;
    T* fc = RES ? U.s_yc + e : fblk + S::fXB + e;
    const T fl = face_h<T>(io, L.s_h + (r + kHalo) * RJ + qq, 1, L.s_vc + r * RJ + qq, 1, side,
                           (side == kW ? 2 : 3) * S::EW + r, L.s_dzy[e], L.s_np, L.s_nh, L.s_ndz, fc, S::FY);
    L.s_Q[e] = fl * L.s_ddx[e];
  }
  __syncthreads();

  // cells: divergence (agrid.py:43-53) and the h update (barotr_pure.py:119-120)
  if (q < nj) {
#pragma unroll
    for (int k = 0; k < S::KC; ++k) {
      const int a = sl + k * S::NS;
      if (a < ni) {
        const int x0 = a * TJ + q, y0 = a * (TJ + 1) + q;
        const T div = L.s_rda[x0] * (L.s_P[x0 + TJ] - L.s_P[x0] + L.s_Q[y0 + 1] - L.s_Q[y0]);
        io.h_out[ov + (a + kHalo) * m] = hpc[k] - div * io.dt;
      }
    }
  }
}

// ---- phase UV -----------------------------------------------------------------
// Phase UV cell and face constants of the tile (cp.async, not yet awaited):
// the tile's prepared block with 16-byte copies when the plan has one for this
// tile shape, else element by element from the constant arrays.
template <typename T, int TI, int TJ, bool FULL>
__device__ __forceinline__ void tile_uv_consts(const Geo<T>& g, const TileBox& b, T* sm) {
  using S = TileShape<TI, TJ>;
  if (g.cblk != nullptr && g.cblk_ti == TI && g.cblk_tj == TJ) {
    constexpr int V = 16 / sizeof(T);
    const T* blk = g.cblk + (long)tile_index<TI, TJ>(b, g.n) * S::cW;
#pragma unroll
    for (int w = threadIdx.x * V; w < S::uConstWords; w += kTileThreads * V) cp_async<16>(sm + S::uG + w, blk + w);
    return;
  }
  const LayoutUV<T, TI, TJ> L(sm);
  const int m = g.m, q = threadIdx.x % TJ, sl = threadIdx.x / TJ;
  const int ni = FULL ? TI : b.ni, nj = FULL ? TJ : b.nj;
  const int o0 = cell32(b.f, b.i0, b.j0 + q, m);
  if (q < nj) {
#pragma unroll
    for (int k = 0; k < S::KC; ++k) {
      const int a = sl + k * S::NS;
      if (a < ni) {
        const int o = o0 + a * m, e = a * TJ + q;
        cp_async_mat(L.s_g + 4 * e, g.gct + 4 * (long)o);
        cp_async_t(L.s_sn + e, g.sina + o);
        cp_async_t(L.s_rda + e, g.rda + o);
        cp_async_t(L.s_rdx + e, g.rdx + o);
        cp_async_t(L.s_rdy + e, g.rdy + o);
        cp_async_t(L.s_af + e, g.a_f + o);
      }
    }
#pragma unroll
    for (int k = 0; k < S::KX; ++k) {
      const int a = sl + k * S::NS;
      if (a <= ni) cp_async_t(L.s_cdy + a * TJ + q, g.c_dy + o0 + a * m);
    }
  }
  if (q <= nj) {
#pragma unroll
    for (int k = 0; k < S::KC; ++k) {
      const int r = sl + k * S::NS;
      if (r < ni) cp_async_t(L.s_ddx + r * (TJ + 1) + q, g.d_dx + o0 + r * m);
    }
  }
  if (nj == TJ && east_row() >= 0 && east_row() < ni) {
    const int r = east_row();
    cp_async_t(L.s_ddx + r * (TJ + 1) + TJ, g.d_dx + cell32(b.f, b.i0 + r, b.j0 + TJ, m));
  }
}

// Phase UV prologue: cell and face constants (cp.async) and the halo-gather descriptors.
template <typename T, int TI, int TJ, bool FULL>
__device__ __forceinline__ void tile_uv_pro_t(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                              Gather<T, TI, TJ, true>& gat, EdgeCnt& cnt, int& P) {
  using S = TileShape<TI, TJ>;
  tile_uv_consts<T, TI, TJ, FULL>(g, b, sm);
  tile_desc<T, TI, TJ, FULL, true, false>(g, io, b, gat, cnt, P, reinterpret_cast<int*>(sm + S::kWordsUV));
}

// RES (tile-resident round): the constants, the face cache and the raw
// velocities of the region are already in shared memory (left there by phase
// H of the same stage), and the stage h of the fb blend is phase H's region h
// (rs.hs); only the new h of the region is read from global memory.
template <typename T, int TI, int TJ, bool FULL, bool RES = false>
__device__ __forceinline__ void tile_uv_main_t(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                               Gather<T, TI, TJ, true, RES>& gat, const EdgeCnt& cnt, int P,
                                               const ResSm<T>& rs = ResSm<T>{}) {
  using S = TileShape<TI, TJ>;
  constexpr int RJ = S::RJ;
  static_assert(6 * TI <= kTileThreads, "one side point per thread");
  const int m = g.m, n = g.n, f = b.f, q = threadIdx.x % TJ, sl = threadIdx.x / TJ;
  const int ni = FULL ? TI : b.ni, nj = FULL ? TJ : b.nj;
  const LayoutUV<T, TI, TJ> L(sm);
  const bool blend = io.beta != T(0.0);  // fb_scheme needs the stage h only when beta_d != 0
  const T* hn_src = (const T*)io.h_out;
  const T* const hb = RES ? rs.hs : L.s_hb;  // stage h of the blend, region layout [RI][RJ]
  const int* const items = RES ? rs.items : reinterpret_cast<const int*>(sm + S::kWordsUV);

  // the tile's face cache block of this stage (written by phase H) -> shared memory, 16 bytes a copy
  if (!RES) {
    constexpr int V = 16 / sizeof(T);
    const T* blk = io.fx + face_block_off<TI, TJ>(b, n);
#pragma unroll
    for (int w = threadIdx.x * V; w < S::fXB; w += kTileThreads * V) cp_async<16>(L.s_xc + w, blk + w);
#pragma unroll
    for (int w = threadIdx.x * V; w < S::fYB; w += kTileThreads * V) cp_async<16>(L.s_yc + w, blk + S::fXB + w);
  }

  // state of the region: interior points by cp.async straight into shared
  // memory (new h, raw v on the vertical bar, raw u on the tile rows and side
  // points, the stage h of the fb blend when beta != 0); halo points that no
  // gather item covers are fetched point by point and stored blended
  T upc[S::KC], vpc[S::KC];
  const EdgeCover ec(b, m);
  const int ov = cell32(f, b.i0 - kHalo, b.j0 + q, m);
#pragma unroll
  for (int k = 0; k < S::KV; ++k) {
    const int r = sl + k * S::NS, i = b.i0 - kHalo + r;
    if (q < nj && r < ni + 6 && (FULL || (i >= kHalo && i < m - kHalo))) {  // halo rows: see below
      const bool row = r >= kHalo && r < ni + kHalo;
      const int e = r * RJ + q + kHalo;
      const int o = ov + r * m;
      cp_async_t(L.s_hn + e, hn_src + o);
      if (!RES) {
        if (blend) cp_async_t(L.s_hb + e, io.h + o);
        cp_async_t(L.s_v + r * TJ + q, io.v + o);
        if (row) cp_async_t(L.s_u + (r - kHalo) * RJ + q + kHalo, io.u + o);
      }
    }
  }
  if (!FULL) {
    // halo rows of the region that no gather item covers (EdgeCover), fetched
    // point by point and stored blended (the new h never has a stored halo)
#pragma unroll 1
    for (int k = 0; k < S::KV; ++k) {
      const int r = sl + k * S::NS, i = b.i0 - kHalo + r;
      if (q < nj && r < ni + 6 && ec.row_staged(i, m) && !(i >= kHalo && i < m - kHalo)) {
        const int e = r * RJ + q + kHalo;
        T hn = fetch_s(hn_src, g, f, i, b.j0 + q, 0);
        if (RES) {  // raw velocities and the stage h staged by phase H
          if (blend) hn = (T(1.0) - io.beta) * hn + io.beta * hb[e];
          L.s_hn[e] = hn;
          continue;
        }
        T u, v;
        fetch_v(io.u, io.v, g, f, i, b.j0 + q, io.stored_halo, u, v);
        if (blend) hn = (T(1.0) - io.beta) * hn + io.beta * fetch_s(io.h, g, f, i, b.j0 + q, io.stored_halo);
        L.s_hn[e] = hn;
        L.s_v[r * TJ + q] = v;
        if (r >= kHalo && r < ni + kHalo) L.s_u[(r - kHalo) * RJ + q + kHalo] = u;
      }
    }
  }
  const int t6 = threadIdx.x;
  const int sr = t6 / 6, sc = t6 - 6 * sr, scc = sc < 3 ? sc : nj + sc, sj = b.j0 - kHalo + scc;
  const bool side_pt = t6 < 6 * ni && (FULL || ec.col_staged(sj, m));
  const bool side_in = FULL || (sj >= kHalo && sj < m - kHalo);
  if (side_pt) {
    const int e = (sr + kHalo) * RJ + scc;
    if (side_in) {
      const int o = cell32(f, b.i0 + sr, sj, m);
      cp_async_t(L.s_hn + e, hn_src + o);
      if (!RES) {
        if (blend) cp_async_t(L.s_hb + e, io.h + o);
        cp_async_t(L.s_u + sr * RJ + scc, io.u + o);
      }
    } else if (RES) {
      T hn = fetch_s(hn_src, g, f, b.i0 + sr, sj, 0);
      if (blend) hn = (T(1.0) - io.beta) * hn + io.beta * hb[e];
      L.s_hn[e] = hn;
    } else {
      T hn = fetch_s(hn_src, g, f, b.i0 + sr, sj, 0), u, v;
      fetch_v(io.u, io.v, g, f, b.i0 + sr, sj, io.stored_halo, u, v);
      if (blend) hn = (T(1.0) - io.beta) * hn + io.beta * fetch_s(io.h, g, f, b.i0 + sr, sj, io.stored_halo);
      L.s_hn[e] = hn;
      L.s_u[sr * RJ + scc] = u;
    }
  }
#pragma unroll
  for (int k = 0; k < S::KC; ++k) {
    const int a = sl + k * S::NS;
    if (q < nj && a < ni) {
      upc[k] = io.up[ov + (a + kHalo) * m];
      vpc[k] = io.vp[ov + (a + kHalo) * m];
    }
  }
  if (!FULL && P > 0) {
    GatherSink<T> sink{L.s_hn, L.s_v, L.s_u, nullptr, nullptr, nullptr};
    sink.hs = hb;
    gat.sources(g, io, b, cnt, P, sink, items);
  }
  cp_async_wait_all();
  __syncthreads();
  if (blend) {  // fb_scheme, barotr_pure.py:52-54, on the points staged by cp.async
#pragma unroll
    for (int k = 0; k < S::KV; ++k) {
      const int r = sl + k * S::NS, i = b.i0 - kHalo + r;
      if (q < nj && r < ni + 6 && (FULL || (i >= kHalo && i < m - kHalo))) {
        const int e = r * RJ + q + kHalo;
        L.s_hn[e] = (T(1.0) - io.beta) * L.s_hn[e] + io.beta * hb[e];
      }
    }
    if (side_pt && side_in) {
      const int e = (sr + kHalo) * RJ + scc;
      L.s_hn[e] = (T(1.0) - io.beta) * L.s_hn[e] + io.beta * hb[e];
    }
    __syncthreads();
  }

  // faces: upwind tangential component (remap.py:73-95) and kinetic energy (barotr_pure.py:91-92)
  if (q < nj) {
#pragma unroll
    for (int k = 0; k < S::KX; ++k) {
      const int a = sl + k * S::NS;
      if (a <= ni) {
        const int e = a * TJ + q;
        const T* pt = L.s_v + a * TJ + q;
        T p6[6];
#pragma unroll
        for (int z = 0; z < 6; ++z) p6[z] = pt[z * TJ];
        const T bc = L.s_xc[e], vis = L.s_xc[S::FX + e];
        const T vt = bc > T(0.0) ? rplus(p6, 1) : rminus(p6 + 1, 1);
        L.s_ku[e] = T(0.5) * (vis * vis + vt * vt);
        L.s_vx[e] = vt * L.s_cdy[e];
      }
    }
  }
#pragma unroll
  for (int k = 0; k <= S::KC; ++k) {
    int r, qq;
    if (k < S::KC) {
      r = sl + k * S::NS;
      qq = q;
      if (r >= ni || q > nj) continue;
    } else {
      r = east_row();
      qq = TJ;
      if (nj != TJ || r < 0 || r >= ni) continue;
    }
    const int e = r * (TJ + 1) + qq;
    const T* pt = L.s_u + r * RJ + qq;
    T p6[6];
#pragma unroll
    for (int z = 0; z < 6; ++z) p6[z] = pt[z];
    const T bc = L.s_yc[e], vis = L.s_yc[S::FY + e];
    const T ut = bc > T(0.0) ? rplus(p6, 1) : rminus(p6 + 1, 1);
    L.s_kv[e] = T(0.5) * (vis * vis + ut * ut);
    L.s_uy[e] = ut * L.s_ddx[e];
  }
  __syncthreads();

  if (q < nj) {
#pragma unroll
    for (int k = 0; k < S::KC; ++k) {
      const int a = sl + k * S::NS;
      if (a >= ni) continue;
      const int e = a * TJ + q;
      const int xf0 = e, xf1 = e + TJ;
      const int yf0 = a * (TJ + 1) + q, yf1 = yf0 + 1;
      const T* G = L.s_g + 4 * e;
      const T u = L.s_u[a * RJ + q + kHalo], v = L.s_v[(a + kHalo) * TJ + q], sn = L.s_sn[e];
      const T uct = (G[0] * u + G[1] * v) * sn, vct = (G[2] * u + G[3] * v) * sn;  // remap.py:34-39
      const T rdx = L.s_rdx[e], rdy = L.s_rdy[e];
      // vorticity (agrid.py:31-41) and advection (barotr_pure.py:78-97)
      const T vort = L.s_rda[e] * (L.s_uy[yf0] + L.s_vx[xf1] - L.s_uy[yf1] - L.s_vx[xf0]);
      const T advx = vort * vct - (L.s_ku[xf1] - L.s_ku[xf0]) * rdx;
      const T advy = -vort * uct - (L.s_kv[yf1] - L.s_kv[yf0]) * rdy;
      // celerity viscosity (barotr_pure.py:63-75) from the cached face fluxes
      const T visx = -(rdx * (L.s_xc[2 * S::FX + xf1] - L.s_xc[2 * S::FX + xf0]));
      const T visy = -(rdy * (L.s_yc[2 * S::FY + yf1] - L.s_yc[2 * S::FY + yf0]));
      // pressure gradient of the new h (agrid.py:55-69, barotr_pure.py:57-60)
      const T* pbx = L.s_hn + (a * RJ + (q + kHalo));
      const T* pby = L.s_hn + ((a + kHalo) * RJ + q);
      T hx[7], hy[7];
#pragma unroll
      for (int z = 0; z < 7; ++z) {
        hx[z] = pbx[z * RJ];
        hy[z] = pby[z];
      }
      const T pgu = T(-9.80) * (rdx * (mid6(hx + 1, 1) - mid6(hx, 1)));
      const T pgv = T(-9.80) * (rdy * (mid6(hy + 1, 1) - mid6(hy, 1)));
      const T af = L.s_af[e];
      // momentum update (barotr_pure.py:149-150)
      const int o = ov + (a + kHalo) * m;
      io.u_out[o] = upc[k] + (pgu + advx + af * vct + visx) * io.dt;
      io.v_out[o] = vpc[k] + (pgv + advy - af * uct + visy) * io.dt;
    }
  }
}

// Tile phases dispatched on the tile's kind: with FP (the full-tile path
// compiled in), full interior tiles run the FULL = true instantiation and the
// others the edge instantiation; without it every tile runs the edge
// instantiation, which handles full tiles too.  The kernel without the full
// path is about half the code: at one-wave sizes (every CTA runs the code
// once, and instruction fetch is the largest stall) it is the faster one.
// Prologue and main part of one tile take the same branch, since both test
// the same tile box.
template <typename T, int TI, int TJ, bool FP = true>
__device__ __forceinline__ void tile_h_pro(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                           Gather<T, TI, TJ, false>& gat, EdgeCnt& cnt, int& P) {
  if (FP && tile_full(b, g.m, TI, TJ))
    tile_h_pro_t<T, TI, TJ, true>(g, io, b, sm, gat, cnt, P);
  else
    tile_h_pro_t<T, TI, TJ, false>(g, io, b, sm, gat, cnt, P);
}
template <typename T, int TI, int TJ, bool FP = true>
__device__ __forceinline__ void tile_h_main(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                            Gather<T, TI, TJ, false>& gat, const EdgeCnt& cnt, int P) {
  if (FP && tile_full(b, g.m, TI, TJ))
    tile_h_main_t<T, TI, TJ, true>(g, io, b, sm, gat, cnt, P);
  else
    tile_h_main_t<T, TI, TJ, false>(g, io, b, sm, gat, cnt, P);
}
template <typename T, int TI, int TJ, bool FP = true>
__device__ __forceinline__ void tile_uv_pro(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                            Gather<T, TI, TJ, true>& gat, EdgeCnt& cnt, int& P) {
  if (FP && tile_full(b, g.m, TI, TJ))
    tile_uv_pro_t<T, TI, TJ, true>(g, io, b, sm, gat, cnt, P);
  else
    tile_uv_pro_t<T, TI, TJ, false>(g, io, b, sm, gat, cnt, P);
}
template <typename T, int TI, int TJ, bool FP = true>
__device__ __forceinline__ void tile_uv_main(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                             Gather<T, TI, TJ, true>& gat, const EdgeCnt& cnt, int P) {
  if (FP && tile_full(b, g.m, TI, TJ))
    tile_uv_main_t<T, TI, TJ, true>(g, io, b, sm, gat, cnt, P);
  else
    tile_uv_main_t<T, TI, TJ, false>(g, io, b, sm, gat, cnt, P);
}

// One tile phase with the prologue issued first (the stream/graph kernels).
template <typename T, int TI, int TJ, bool FP = true>
__device__ __forceinline__ void tile_h(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm) {
  Gather<T, TI, TJ, false> gat;
  EdgeCnt cnt;
  int P;
  tile_h_pro<T, TI, TJ, FP>(g, io, b, sm, gat, cnt, P);
  wait_prior_grid();
  tile_h_main<T, TI, TJ, FP>(g, io, b, sm, gat, cnt, P);
}
template <typename T, int TI, int TJ, bool FP = true>
__device__ __forceinline__ void tile_uv(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm) {
  Gather<T, TI, TJ, true> gat;
  EdgeCnt cnt;
  int P;
  tile_uv_pro<T, TI, TJ, FP>(g, io, b, sm, gat, cnt, P);
  wait_prior_grid();
  tile_uv_main<T, TI, TJ, FP>(g, io, b, sm, gat, cnt, P);
}


// ---------------------------------------------------------------------------
// Grid-wide barrier of the persistent round kernel
// ---------------------------------------------------------------------------
// Monotone arrival counter: the k-th barrier completes when the low 31 bits
// of the counter reach k * gridDim.x.  Thread 0 of each CTA arrives with a
// release reduction (publishing the CTA's writes, ordered by the preceding
// __syncthreads) and polls with acquire loads, at most ``limit`` times.  A CTA
// that gives up raises kErrBarrierTimeout and sets the counter's top bit, which
// every other CTA sees at its next poll: all CTAs then leave the round.
// Returns false when the round must stop.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned& gen, int* err, long long limit) {
  __shared__ int s_ok;
  constexpr unsigned kAbort = 0x80000000u;
  __syncthreads();
  if (threadIdx.x == 0) {
    ++gen;
    const unsigned target = gen * gridDim.x;
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    long long polls = 0;
    int ok = 1;
    while (true) {
      unsigned seen;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(bar) : "memory");
      if (seen & kAbort) {
        ok = 0;
        break;
      }
      if ((int)((seen & ~kAbort) - target) >= 0) break;
      if (++polls > limit) {
        atomicOr(err, kErrBarrierTimeout);
        atomicOr(bar, kAbort);
        ok = 0;
        break;
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Stage pointers of (substep, stage) of a round, ``step`` counted from the
// round's first substep; mirrors the host schedule.
// Fields are picked with constant indexes only, so the kernel arguments are
// never addressed (which would copy them to local memory).
template <typename T>
__device__ __forceinline__ StageIO<T> round_stage(const RoundArgs<T>& a, int step, int st) {
  StageIO<T> io;
  const int nst = a.rk == 2 ? 2 : 3;
  const bool first = step == 0, last = st == nst - 1;
  // stage input: the round input (first substep) or the running state, then Y, then Z
  io.h = st == 0 ? (first ? a.x0[0] : a.x[0]) : (st == 1 ? a.y[0] : a.z[0]);
  io.u = st == 0 ? (first ? a.x0[1] : a.x[1]) : (st == 1 ? a.y[1] : a.z[1]);
  io.v = st == 0 ? (first ? a.x0[2] : a.x[2]) : (st == 1 ? a.y[2] : a.z[2]);
  io.hp = first ? a.b0[0] : a.x[0];
  io.up = first ? a.b0[1] : a.x[1];
  io.vp = first ? a.b0[2] : a.x[2];
  io.h_out = last ? a.x[0] : (st == 0 ? a.y[0] : a.z[0]);
  io.u_out = last ? a.x[1] : (st == 0 ? a.y[1] : a.z[1]);
  io.v_out = last ? a.x[2] : (st == 0 ? a.y[2] : a.z[2]);
  io.fx = a.fx;
  double dt;
  if (a.rk == 2) {
    dt = st == 0 ? a.dtb / 2.0 : a.dtb;      // barotr.py:50-56
    io.beta = T(0.0);
  } else {
    dt = st == 0 ? a.dtb / 3.0 : (st == 1 ? a.dtb / 2.0 : a.dtb);  // barotr.py:73-83
    io.beta = T(1.0);
  }
  io.dt = (T)dt;
  io.stored_halo = (first && st == 0) ? 1 : 0;
  io.last = last ? 1 : 0;
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
