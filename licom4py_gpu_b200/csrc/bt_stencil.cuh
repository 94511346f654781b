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
// A CTA of kTileThreads threads computes one TI x TJ tile of one face.  Its
// stencil region (the tile plus 3 cells on each side, without the region
// corners) is staged into shared memory with cp.async, so every global load
// of the region is in flight at once; halo cells of the region are gathered
// (two-level chain: descriptor, then sources), the neighbouring face's edge
// values are recomputed, and per-cell / per-face constants are prefetched into
// registers, all before the first barrier.
constexpr int kTileThreads = 256;

template <int TI, int TJ>
struct TileShape {
  static constexpr int RI = TI + 6, RJ = TJ + 6, R = RI * RJ;
  static constexpr int FX = (TI + 1) * TJ;   // x faces
  static constexpr int FY = TI * (TJ + 1);   // y faces
  static constexpr int EW = TI > TJ ? TI : TJ;
  static constexpr int NE = 4 * EW;          // edge slots: 4 kinds x max(TI, TJ) positions
  static constexpr int NIT = (R + kTileThreads - 1) / kTileThreads;
  static constexpr int CIT = (TI * TJ + kTileThreads - 1) / kTileThreads;
  static constexpr int FIT = (FX + FY + kTileThreads - 1) / kTileThreads;
  static constexpr int C = TI * TJ;
  // region: h, u, v, g(4), s, uc, vc [+ hn for UV]; face and cell arrays;
  // neighbour edge lines (6 contravariant values + 6 h values + depth per slot)
  static constexpr int kWordsH = 10 * R + 3 * FX + 3 * FY + 2 * C + 13 * NE;
  // UV: cells g(4), s, rda, rdx, rdy, af, up, vp; region u, v, hn, h; faces:
  // cache (3) + kinetic energy + tangential + c_dy / d_dx
  static constexpr int kWordsUV = 11 * C + 4 * R + 6 * FX + 6 * FY;
  static constexpr int MI = 4;               // gather items per thread handled in the two-sweep path
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
template <typename T>
__device__ __forceinline__ T pull_s(const Pull<T>& p, const T* F) {
  return p.w0 * F[p.s.x] + p.w1 * F[p.s.y];
}
template <typename T>
__device__ __forceinline__ void pull_v(const Pull<T>& p, const Geo<T>& g, const T* U, const T* V, long o,
                                       T& u, T& v) {
  const T* C0 = g.c2l + 4 * (long)p.s.x;
  const T* C1 = g.c2l + 4 * (long)p.s.y;
  const T u0 = U[p.s.x], v0 = V[p.s.x], u1 = U[p.s.y], v1 = V[p.s.y];
  const T ull0 = C0[0] * u0 + C0[1] * v0, vll0 = C0[2] * u0 + C0[3] * v0;
  const T ull1 = C1[0] * u1 + C1[1] * v1, vll1 = C1[2] * u1 + C1[3] * v1;
  const T ull = p.w0 * ull0 + p.w1 * ull1;
  const T vll = p.w0 * vll0 + p.w1 * vll1;
  const T* L = g.l2c + 4 * o;
  u = L[0] * ull + L[1] * vll;
  v = L[2] * ull + L[3] * vll;
}

// ---- the tile's face-edge positions ----------------------------------------
// Item q of a tile's edge list: kind 0/1 = x faces of side S/N (position along
// the tile's columns), kind 2/3 = y faces of side W/E (along the tile's rows).
struct EdgeItem {
  int kind, pos, side, k;
};
__device__ __forceinline__ int edge_count(const TileBox& b, int m, int* cnt) {
  cnt[0] = b.i0 == kHalo ? b.nj : 0;
  cnt[1] = b.i0 + b.ni == m - kHalo ? b.nj : 0;
  cnt[2] = b.j0 == kHalo ? b.ni : 0;
  cnt[3] = b.j0 + b.nj == m - kHalo ? b.ni : 0;
  return cnt[0] + cnt[1] + cnt[2] + cnt[3];
}
__device__ __forceinline__ EdgeItem edge_item(const TileBox& b, const int* cnt, int q) {
  EdgeItem e;
  int kind = 0;
  while (q >= cnt[kind]) q -= cnt[kind++];
  e.kind = kind;
  e.pos = q;
  const int sides[4] = {kS, kN, kW, kE};
  e.side = sides[kind];
  e.k = kind < 2 ? (b.j0 + q - kHalo) : (b.i0 + q - kHalo);
  return e;
}

// Work items of a tile that touches face edges, spread over the whole CTA:
//   item t < 3P:  halo cell at depth t % 3 outside edge position t / 3 of the
//                 tile (its h, u, v when the stored halo is not valid, and the
//                 new h in phase UV) -- a gather from the neighbouring face;
//   item t >= 3P: point q = (t - 3P) % 6 of the neighbour's 6-point line normal
//                 to the shared edge at position (t - 3P) / 6: its contravariant
//                 normal velocity (and h for the mass-flux average).
// P is the number of edge positions of the tile.  Descriptor loads of all
// items go out in a first sweep, source loads in a second, so a CTA waits for
// two L2 round trips instead of one chain per point.
struct ItemCell {
  int f, i, j;      // cell whose value the item needs
  int slot;         // region index (region items) or edge slot*6 + q (line items)
  int line, y, q;   // line item: 1, normal axis (1 = y), point index
};

__device__ __forceinline__ ItemCell decode_item(const TileBox& b, const int* cnt, int P, int t, int m, int n,
                                                const int* route, int RJ, int EW) {
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
    c.slot = r * RJ + cc;
    c.line = 0;
    c.y = 0;
    c.q = 0;
  } else {
    const int t2 = t - 3 * P;
    const EdgeItem e = edge_item(b, cnt, t2 / 6);
    const int q = t2 % 6;
    const int r = route[b.f * 4 + e.side];
    const int ns = route_side(r);
    const int kk = route_rev(r) ? n - 1 - e.k : e.k;
    c.f = route_nb(r);
    edge_point(ns, kk, q, m, c.i, c.j);
    c.slot = (e.kind * EW + e.pos) * 6 + q;
    c.line = 1;
    c.y = (ns == kE || ns == kW);
    c.q = q;
  }
  return c;
}

template <typename T, int TI, int TJ, bool UV>
struct Gather {
  using S = TileShape<TI, TJ>;
  // phase H gathers the region halo and the neighbour edge lines (9 items per
  // edge position); phase UV only the region halo (3 per position)
  static constexpr int kPerPos = UV ? 3 : 9;
  Pull<T> pd[S::MI];
  bool pl[S::MI];

  __device__ __forceinline__ static bool needs_pull(const StageIO<T>& io, const ItemCell& c, int m) {
    return !is_interior(c.i, c.j, m) && (!io.stored_halo || (UV && !c.line));
  }

  // sweep 1: descriptors of the items' halo gathers (constants, may precede the grid dependency)
  __device__ __forceinline__ void descriptors(const Geo<T>& g, const StageIO<T>& io, const TileBox& b,
                                              const int* cnt, int P) {
    const int nitems = kPerPos * P;
#pragma unroll
    for (int k = 0; k < S::MI; ++k) {
      const int t = threadIdx.x + k * kTileThreads;
      pl[k] = false;
      if (t < nitems) {
        const ItemCell c = decode_item(b, cnt, P, t, g.m, g.n, g.route, S::RJ, S::EW);
        if (needs_pull(io, c, g.m)) {
          pd[k] = pull_desc(g, c.f, c.i, c.j);
          pl[k] = true;
        }
      }
    }
  }

  __device__ __forceinline__ void one(const Geo<T>& g, const StageIO<T>& io, const ItemCell& c, const Pull<T>& p,
                                      bool pull, T* s_h, T* s_u, T* s_v, T* s_hn, T* s_np, T* s_nh, T* s_ndz) {
    const bool want_h = !UV && io.last;  // neighbour h for the mass-flux average
    const long o = cell(c.f, c.i, c.j, g.m);
    if (!c.line) {
      if (!io.stored_halo) {  // stored halos are staged by cp.async
        T u, v;
        pull_v(p, g, io.u, io.v, o, u, v);
        s_h[c.slot] = pull_s(p, io.h);
        s_u[c.slot] = u;
        s_v[c.slot] = v;
      }
      if (UV) s_hn[c.slot] = pull_s(p, (const T*)io.h_out);
    } else {
      T u, v, h = T(0.0);
      if (pull) {
        pull_v(p, g, io.u, io.v, o, u, v);
        if (want_h) h = pull_s(p, io.h);
      } else {
        u = io.u[o];
        v = io.v[o];
        if (want_h) h = io.h[o];
      }
      s_np[c.slot] = contra(g, o, u, v, c.y);
      if (want_h) {
        s_nh[c.slot] = h;
        if (c.q == 3) s_ndz[c.slot / 6] = c.y ? g.dzph_y[o] : g.dzph_x[o];
      }
    }
  }

  // sweep 2: sources (state, after the grid dependency) and the items' values
  __device__ __forceinline__ void sources(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, const int* cnt,
                                          int P, T* s_h, T* s_u, T* s_v, T* s_hn, T* s_np, T* s_nh, T* s_ndz) {
    const int nitems = kPerPos * P;
#pragma unroll
    for (int k = 0; k < S::MI; ++k) {
      const int t = threadIdx.x + k * kTileThreads;
      if (t < nitems) {
        const ItemCell c = decode_item(b, cnt, P, t, g.m, g.n, g.route, S::RJ, S::EW);
        one(g, io, c, pd[k], pl[k], s_h, s_u, s_v, s_hn, s_np, s_nh, s_ndz);
      }
    }
    // items beyond MI per thread (only tiles spanning several face edges of tiny faces)
    for (int t = threadIdx.x + S::MI * kTileThreads; t < nitems; t += kTileThreads) {
      const ItemCell c = decode_item(b, cnt, P, t, g.m, g.n, g.route, S::RJ, S::EW);
      const bool pull = needs_pull(io, c, g.m);
      Pull<T> p;
      if (pull) p = pull_desc(g, c.f, c.i, c.j);
      one(g, io, c, p, pull, s_h, s_u, s_v, s_hn, s_np, s_nh, s_ndz);
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

// Constants of the tile's faces and cells, staged by cp.async before the
// state: depth and c_dy on x faces, depth and d_dx on y faces, and per cell
// rda (+ rdx, rdy, a_f for phase UV).
template <typename T, int TI, int TJ, bool UV>
__device__ __forceinline__ void stage_consts(const Geo<T>& g, const TileBox& b, T* s_dzx, T* s_cdy, T* s_dzy,
                                             T* s_ddx, T* s_rda, T* s_rdx, T* s_rdy, T* s_af) {
  using S = TileShape<TI, TJ>;
  const int m = g.m, f = b.f, tid = threadIdx.x;
  for (int e = tid; e < S::FX + S::FY; e += kTileThreads) {
    if (e < S::FX) {
      const int a = e / TJ, q = e % TJ;
      if (a > b.ni || q >= b.nj) continue;
      const long o = cell(f, b.i0 + a, b.j0 + q, m);
      cp_async_t(s_dzx + e, g.dzph_x + o);
      cp_async_t(s_cdy + e, g.c_dy + o);
    } else {
      const int e2 = e - S::FX, a = e2 / (TJ + 1), q = e2 % (TJ + 1);
      if (a >= b.ni || q > b.nj) continue;
      const long o = cell(f, b.i0 + a, b.j0 + q, m);
      cp_async_t(s_dzy + e2, g.dzph_y + o);
      cp_async_t(s_ddx + e2, g.d_dx + o);
    }
  }
  for (int e = tid; e < S::C; e += kTileThreads) {
    const int a = e / TJ, q = e % TJ;
    if (a >= b.ni || q >= b.nj) continue;
    const long o = cell(f, b.i0 + a, b.j0 + q, m);
    cp_async_t(s_rda + e, g.rda + o);
    if (UV) {
      cp_async_t(s_rdx + e, g.rdx + o);
      cp_async_t(s_rdy + e, g.rdy + o);
      cp_async_t(s_af + e, g.a_f + o);
    }
  }
}

// gct and sina of the region (constants).
template <typename T, int TI, int TJ>
__device__ __forceinline__ void stage_region_consts(const Geo<T>& g, const TileBox& b, T* s_g, T* s_s) {
  using S = TileShape<TI, TJ>;
  constexpr int RJ = S::RJ;
#pragma unroll
  for (int it = 0; it < S::NIT; ++it) {
    const int e = threadIdx.x + it * kTileThreads;
    if (e >= S::R) break;
    const int r = e / RJ, c = e - r * RJ;
    if (!region_needed(r, c, b.ni, b.nj)) continue;
    const long o = cell(b.f, b.i0 - kHalo + r, b.j0 - kHalo + c, g.m);
    cp_async_mat(s_g + 4 * e, g.gct + 4 * o);
    cp_async_t(s_s + e, g.sina + o);
  }
}

// State of the region: h, u, v (interior cells, or every cell when the stored
// halo is valid) and the new h of interior cells when HN.
template <typename T, int TI, int TJ, bool HN>
__device__ __forceinline__ void stage_region_state(const Geo<T>& g, const StageIO<T>& io, const TileBox& b,
                                                   T* s_h, T* s_u, T* s_v, T* s_hn) {
  using S = TileShape<TI, TJ>;
  constexpr int RJ = S::RJ;
  const int m = g.m;
  const T* hn_src = (const T*)io.h_out;
#pragma unroll
  for (int it = 0; it < S::NIT; ++it) {
    const int e = threadIdx.x + it * kTileThreads;
    if (e >= S::R) break;
    const int r = e / RJ, c = e - r * RJ;
    if (!region_needed(r, c, b.ni, b.nj)) continue;
    const int i = b.i0 - kHalo + r, j = b.j0 - kHalo + c;
    const long o = cell(b.f, i, j, m);
    const bool inner = is_interior(i, j, m);
    if (io.stored_halo || inner) {
      cp_async_t(s_h + e, io.h + o);
      cp_async_t(s_u + e, io.u + o);
      cp_async_t(s_v + e, io.v + o);
    }
    if (HN && inner) cp_async_t(s_hn + e, hn_src + o);
  }
}

// Shared-memory layout of phase H (offsets in words).
template <typename T, int TI, int TJ>
struct LayoutH {
  using S = TileShape<TI, TJ>;
  T *s_h, *s_u, *s_v, *s_g, *s_s, *s_uc, *s_vc, *s_fu, *s_fv, *s_dzx, *s_cdy, *s_dzy, *s_ddx, *s_rda, *s_hp,
      *s_np, *s_nh, *s_ndz;
  __device__ __forceinline__ explicit LayoutH(T* sm) {
    s_h = sm;
    s_u = s_h + S::R;
    s_v = s_u + S::R;
    s_g = s_v + S::R;      // [R][4]
    s_s = s_g + 4 * S::R;
    s_uc = s_s + S::R;
    s_vc = s_uc + S::R;
    s_fu = s_vc + S::R;    // [TI+1][TJ] mass flux on x faces
    s_fv = s_fu + S::FX;   // [TI][TJ+1] on y faces
    s_dzx = s_fv + S::FY;  // [TI+1][TJ]
    s_cdy = s_dzx + S::FX;
    s_dzy = s_cdy + S::FX; // [TI][TJ+1]
    s_ddx = s_dzy + S::FY;
    s_rda = s_ddx + S::FY; // [TI][TJ]
    s_hp = s_rda + S::C;
    s_np = s_hp + S::C;    // [NE][6] neighbour line: contravariant normal velocity
    s_nh = s_np + 6 * S::NE;   // [NE][6] neighbour line: h
    s_ndz = s_nh + 6 * S::NE;  // [NE] neighbour depth at the edge face
  }
};

// Phase H prologue: constants of the tile (cp.async, not yet awaited) and the
// halo-gather descriptors.  Independent of the state, so it may run before the
// previous phase has finished (programmatic launch, or before a grid barrier).
template <typename T, int TI, int TJ>
__device__ __forceinline__ void tile_h_pro(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                           Gather<T, TI, TJ, false>& gat, int* cnt, int& P) {
  const LayoutH<T, TI, TJ> L(sm);
  stage_region_consts<T, TI, TJ>(g, b, L.s_g, L.s_s);
  stage_consts<T, TI, TJ, false>(g, b, L.s_dzx, L.s_cdy, L.s_dzy, L.s_ddx, L.s_rda, nullptr, nullptr, nullptr);
  P = edge_count(b, g.m, cnt);
  if (P > 0) gat.descriptors(g, io, b, cnt, P);
}

// Phase H of one tile: writes the new h on the tile's interior cells.
template <typename T, int TI, int TJ>
__device__ void tile_h_main(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                            Gather<T, TI, TJ, false>& gat, const int* cnt, int P) {
  using S = TileShape<TI, TJ>;
  constexpr int RJ = S::RJ;
  const int m = g.m, f = b.f, tid = threadIdx.x;
  const LayoutH<T, TI, TJ> L(sm);
  T* s_h = L.s_h;
  T *s_u = L.s_u, *s_v = L.s_v, *s_g = L.s_g, *s_s = L.s_s, *s_uc = L.s_uc, *s_vc = L.s_vc;
  T *s_fu = L.s_fu, *s_fv = L.s_fv, *s_dzx = L.s_dzx, *s_cdy = L.s_cdy, *s_dzy = L.s_dzy, *s_ddx = L.s_ddx;
  T *s_rda = L.s_rda, *s_hp = L.s_hp, *s_np = L.s_np, *s_nh = L.s_nh, *s_ndz = L.s_ndz;
  stage_region_state<T, TI, TJ, false>(g, io, b, s_h, s_u, s_v, nullptr);
  for (int e = tid; e < S::C; e += kTileThreads) {
    const int a = e / TJ, q = e % TJ;
    if (a < b.ni && q < b.nj) cp_async_t(s_hp + e, io.hp + cell(f, b.i0 + a, b.j0 + q, m));
  }
  if (P > 0) gat.sources(g, io, b, cnt, P, s_h, s_u, s_v, nullptr, s_np, s_nh, s_ndz);
  cp_async_wait_all();
  __syncthreads();

  // contravariant velocities on the region (remap.py:34-39)
#pragma unroll
  for (int it = 0; it < S::NIT; ++it) {
    const int e = tid + it * kTileThreads;
    if (e >= S::R) break;
    const int r = e / RJ, c = e - r * RJ;
    if (!region_needed(r, c, b.ni, b.nj)) continue;
    const T* G = s_g + 4 * e;
    const T u = s_u[e], v = s_v[e], sn = s_s[e];
    s_uc[e] = (G[0] * u + G[1] * v) * sn;
    s_vc[e] = (G[2] * u + G[3] * v) * sn;
  }
  __syncthreads();

  // faces: x faces i = i0..i0+ni on the tile's columns, then y faces j = j0..j0+nj on its rows
  for (int e = tid; e < S::FX + S::FY; e += kTileThreads) {
    const bool xf = e < S::FX;
    int a, q, stride, base, side, kind, pos, fi;
    if (xf) {
      a = e / TJ;
      q = e % TJ;
      if (a > b.ni || q >= b.nj) continue;
      stride = RJ;
      base = a * RJ + (q + kHalo);
      side = xface_side(b.i0 + a, m);
      kind = side == kS ? 0 : 1;
      pos = q;
      fi = e;
    } else {
      fi = e - S::FX;
      a = fi / (TJ + 1);
      q = fi % (TJ + 1);
      if (a >= b.ni || q > b.nj) continue;
      stride = 1;
      base = (a + kHalo) * RJ + q;
      side = yface_side(b.j0 + q, m);
      kind = side == kW ? 2 : 3;
      pos = a;
    }
    const T* ph = s_h + base;
    const T* pu = (xf ? s_uc : s_vc) + base;
    const T ue = rplus(pu, stride), uw = rminus(pu + stride, stride);
    T bc = T(0.5) * (ue + uw);
    const int slot = kind * S::EW + pos;
    if (side >= 0) bc = (bc + line_raw(s_np + 6 * slot)) / T(2.0);
    const T dz = xf ? s_dzx[fi] : s_dzy[fi];
    const T he = rplus(ph, stride), hw = rminus(ph + stride, stride);
    const T cc = celerity(mid6(ph, stride), dz);
    const T vis = bc + (T(4.9) / cc) * (he - hw);
    T fl = dz * vis + (vis > T(0.0) ? he : hw) * vis;
    if (io.last && side >= 0) {  // the neighbour's flux at the same edge face (barotr_pure.py:29-49)
      const T* nh = s_nh + 6 * slot;
      const T ndz = s_ndz[slot];
      const T nhe = rplus(nh, 1), nhw = rminus(nh + 1, 1);
      const T nc = celerity(mid6(nh, 1), ndz);
      const T nvis = bc + (T(4.9) / nc) * (nhe - nhw);
      fl = (fl + (ndz * nvis + (nvis > T(0.0) ? nhe : nhw) * nvis)) / T(2.0);
    }
    // face cache for phase UV: each face is written by the one tile that owns it
    const int n = g.n;
    T* fc;
    if (xf) {
      s_fu[fi] = fl;
      fc = (a < b.ni || b.i0 + b.ni == m - kHalo)
               ? io.fx + 3 * (((long)f * (n + 1) + (b.i0 - kHalo + a)) * n + (b.j0 - kHalo + q))
               : nullptr;
    } else {
      s_fv[fi] = fl;
      fc = (q < b.nj || b.j0 + b.nj == m - kHalo)
               ? io.fy + 3 * (((long)f * n + (b.i0 - kHalo + a)) * (n + 1) + (b.j0 - kHalo + q))
               : nullptr;
    }
    if (fc) {
      fc[0] = bc;
      fc[1] = vis;
      fc[2] = T(0.5) * cc * (ue - uw);   // celerity viscosity flux, barotr_pure.py:68-69
    }
  }
  __syncthreads();

  // cells: divergence (agrid.py:43-53) and the h update (barotr_pure.py:119-120)
  for (int e = tid; e < S::C; e += kTileThreads) {
    const int a = e / TJ, q = e % TJ;
    if (a >= b.ni || q >= b.nj) continue;
    const long o = cell(f, b.i0 + a, b.j0 + q, m);
    const int x0 = e, x1 = e + TJ;
    const int y0 = a * (TJ + 1) + q, y1 = y0 + 1;
    const T div = s_rda[x0] * (s_fu[x1] * s_cdy[x1] - s_fu[x0] * s_cdy[x0] + s_fv[y1] * s_ddx[y1] -
                               s_fv[y0] * s_ddx[y0]);
    io.h_out[o] = s_hp[x0] - div * io.dt;
  }
}

// Phase UV of one tile: writes the new u, v on the tile's interior cells.
// io.h_out must hold the new h of every face (interior) and io.fx / io.fy the
// face cache of this stage, both from phase H.
template <typename T, int TI, int TJ>
struct LayoutUV {
  using S = TileShape<TI, TJ>;
  T *s_g, *s_s, *s_rda, *s_rdx, *s_rdy, *s_af, *s_up, *s_vp, *s_u, *s_v, *s_hn, *s_h, *s_xc, *s_ku, *s_vx,
      *s_cdy, *s_yc, *s_kv, *s_uy, *s_ddx;
  __device__ __forceinline__ explicit LayoutUV(T* sm) {
    s_g = sm;              // cells [C][4] gct (16-byte aligned for cp.async)
    s_s = s_g + 4 * S::C;  // cells: sina
    s_rda = s_s + S::C;
    s_rdx = s_rda + S::C;
    s_rdy = s_rdx + S::C;
    s_af = s_rdy + S::C;
    s_up = s_af + S::C;
    s_vp = s_up + S::C;
    s_u = s_vp + S::C;     // region: raw u, v, new h (then the blended h), stage h
    s_v = s_u + S::R;
    s_hn = s_v + S::R;
    s_h = s_hn + S::R;
    s_xc = s_h + S::R;     // x faces [TI+1][TJ]: cache (3), kinetic energy, tangential v, c_dy
    s_ku = s_xc + 3 * S::FX;
    s_vx = s_ku + S::FX;
    s_cdy = s_vx + S::FX;
    s_yc = s_cdy + S::FX;  // y faces [TI][TJ+1]: cache (3), kinetic energy, tangential u, d_dx
    s_kv = s_yc + 3 * S::FY;
    s_uy = s_kv + S::FY;
    s_ddx = s_uy + S::FY;
  }
};

// Phase UV prologue: cell and face constants (cp.async) and the halo-gather descriptors.
template <typename T, int TI, int TJ>
__device__ __forceinline__ void tile_uv_pro(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                                            Gather<T, TI, TJ, true>& gat, int* cnt, int& P) {
  using S = TileShape<TI, TJ>;
  const LayoutUV<T, TI, TJ> L(sm);
  const int m = g.m, f = b.f, tid = threadIdx.x;
  for (int e = tid; e < S::C; e += kTileThreads) {
    const int a = e / TJ, q = e % TJ;
    if (a >= b.ni || q >= b.nj) continue;
    const long o = cell(f, b.i0 + a, b.j0 + q, m);
    cp_async_mat(L.s_g + 4 * e, g.gct + 4 * o);
    cp_async_t(L.s_s + e, g.sina + o);
    cp_async_t(L.s_rda + e, g.rda + o);
    cp_async_t(L.s_rdx + e, g.rdx + o);
    cp_async_t(L.s_rdy + e, g.rdy + o);
    cp_async_t(L.s_af + e, g.a_f + o);
  }
  for (int e = tid; e < S::FX + S::FY; e += kTileThreads) {
    if (e < S::FX) {
      const int a = e / TJ, q = e % TJ;
      if (a <= b.ni && q < b.nj) cp_async_t(L.s_cdy + e, g.c_dy + cell(f, b.i0 + a, b.j0 + q, m));
    } else {
      const int e2 = e - S::FX, a = e2 / (TJ + 1), q = e2 % (TJ + 1);
      if (a < b.ni && q <= b.nj) cp_async_t(L.s_ddx + e2, g.d_dx + cell(f, b.i0 + a, b.j0 + q, m));
    }
  }
  P = edge_count(b, m, cnt);
  if (P > 0) gat.descriptors(g, io, b, cnt, P);
}

template <typename T, int TI, int TJ>
__device__ void tile_uv_main(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm,
                             Gather<T, TI, TJ, true>& gat, const int* cnt, int P) {
  using S = TileShape<TI, TJ>;
  constexpr int RJ = S::RJ;
  const int m = g.m, n = g.n, f = b.f, tid = threadIdx.x;
  const LayoutUV<T, TI, TJ> L(sm);
  T *s_g = L.s_g, *s_s = L.s_s, *s_rda = L.s_rda, *s_rdx = L.s_rdx, *s_rdy = L.s_rdy, *s_af = L.s_af;
  T *s_up = L.s_up, *s_vp = L.s_vp, *s_u = L.s_u, *s_v = L.s_v, *s_hn = L.s_hn, *s_h = L.s_h;
  T *s_xc = L.s_xc, *s_ku = L.s_ku, *s_vx = L.s_vx, *s_cdy = L.s_cdy, *s_yc = L.s_yc, *s_kv = L.s_kv;
  T *s_uy = L.s_uy, *s_ddx = L.s_ddx;
  const bool blend = io.beta != T(0.0);  // fb_scheme needs the stage h only when beta_d != 0

  // state: region u, v, new h (and h), cells' base velocities, the face cache
  const T* hn_src = (const T*)io.h_out;
#pragma unroll
  for (int it = 0; it < S::NIT; ++it) {
    const int e = tid + it * kTileThreads;
    if (e >= S::R) break;
    const int r = e / RJ, c = e - r * RJ;
    if (!region_needed(r, c, b.ni, b.nj)) continue;
    const int i = b.i0 - kHalo + r, j = b.j0 - kHalo + c;
    const long o = cell(f, i, j, m);
    const bool inner = is_interior(i, j, m);
    if (io.stored_halo || inner) {
      cp_async_t(s_u + e, io.u + o);
      cp_async_t(s_v + e, io.v + o);
      if (blend) cp_async_t(s_h + e, io.h + o);
    }
    if (inner) cp_async_t(s_hn + e, hn_src + o);
  }
  for (int e = tid; e < S::C; e += kTileThreads) {
    const int a = e / TJ, q = e % TJ;
    if (a >= b.ni || q >= b.nj) continue;
    const long o = cell(f, b.i0 + a, b.j0 + q, m);
    cp_async_t(s_up + e, io.up + o);
    cp_async_t(s_vp + e, io.vp + o);
  }
  for (int e = tid; e < S::FX + S::FY; e += kTileThreads) {
    const T* src;
    T* dst;
    if (e < S::FX) {
      const int a = e / TJ, q = e % TJ;
      if (a > b.ni || q >= b.nj) continue;
      src = io.fx + 3 * (((long)f * (n + 1) + (b.i0 - kHalo + a)) * n + (b.j0 - kHalo + q));
      dst = s_xc + 3 * e;
    } else {
      const int e2 = e - S::FX, a = e2 / (TJ + 1), q = e2 % (TJ + 1);
      if (a >= b.ni || q > b.nj) continue;
      src = io.fy + 3 * (((long)f * n + (b.i0 - kHalo + a)) * (n + 1) + (b.j0 - kHalo + q));
      dst = s_yc + 3 * e2;
    }
    cp_async_t(dst, src);
    cp_async_t(dst + 1, src + 1);
    cp_async_t(dst + 2, src + 2);
  }
  if (P > 0) gat.sources(g, io, b, cnt, P, s_h, s_u, s_v, s_hn, nullptr, nullptr, nullptr);
  cp_async_wait_all();
  __syncthreads();

  if (blend) {
#pragma unroll
    for (int it = 0; it < S::NIT; ++it) {
      const int e = tid + it * kTileThreads;
      if (e >= S::R) break;
      const int r = e / RJ, c = e - r * RJ;
      if (!region_needed(r, c, b.ni, b.nj)) continue;
      s_hn[e] = (T(1.0) - io.beta) * s_hn[e] + io.beta * s_h[e];  // fb_scheme, barotr_pure.py:52-54
    }
  }
  // faces: upwind tangential component (remap.py:73-95) and kinetic energy (barotr_pure.py:91-92)
  for (int e = tid; e < S::FX + S::FY; e += kTileThreads) {
    if (e < S::FX) {
      const int a = e / TJ, q = e % TJ;
      if (a > b.ni || q >= b.nj) continue;
      const T* pt = s_v + a * RJ + (q + kHalo);
      const T* c = s_xc + 3 * e;
      const T vt = c[0] > T(0.0) ? rplus(pt, RJ) : rminus(pt + RJ, RJ);
      s_ku[e] = T(0.5) * (c[1] * c[1] + vt * vt);
      s_vx[e] = vt;
    } else {
      const int e2 = e - S::FX, a = e2 / (TJ + 1), q = e2 % (TJ + 1);
      if (a >= b.ni || q > b.nj) continue;
      const T* pt = s_u + (a + kHalo) * RJ + q;
      const T* c = s_yc + 3 * e2;
      const T ut = c[0] > T(0.0) ? rplus(pt, 1) : rminus(pt + 1, 1);
      s_kv[e2] = T(0.5) * (c[1] * c[1] + ut * ut);
      s_uy[e2] = ut;
    }
  }
  __syncthreads();

  for (int e = tid; e < S::C; e += kTileThreads) {
    const int a = e / TJ, q = e % TJ;
    if (a >= b.ni || q >= b.nj) continue;
    const long o = cell(f, b.i0 + a, b.j0 + q, m);
    const int xf0 = e, xf1 = e + TJ;
    const int yf0 = a * (TJ + 1) + q, yf1 = yf0 + 1;
    const int lc = (a + kHalo) * RJ + (q + kHalo);
    const T* G = s_g + 4 * e;
    const T u = s_u[lc], v = s_v[lc], sn = s_s[e];
    const T uct = (G[0] * u + G[1] * v) * sn, vct = (G[2] * u + G[3] * v) * sn;  // remap.py:34-39
    const T rdx = s_rdx[e], rdy = s_rdy[e];
    // vorticity (agrid.py:31-41) and advection (barotr_pure.py:78-97)
    const T vort = s_rda[e] * (s_uy[yf0] * s_ddx[yf0] + s_vx[xf1] * s_cdy[xf1] - s_uy[yf1] * s_ddx[yf1] -
                               s_vx[xf0] * s_cdy[xf0]);
    const T advx = vort * vct - (s_ku[xf1] - s_ku[xf0]) * rdx;
    const T advy = -vort * uct - (s_kv[yf1] - s_kv[yf0]) * rdy;
    // celerity viscosity (barotr_pure.py:63-75) from the cached face fluxes
    const T visx = -(rdx * (s_xc[3 * xf1 + 2] - s_xc[3 * xf0 + 2]));
    const T visy = -(rdy * (s_yc[3 * yf1 + 2] - s_yc[3 * yf0 + 2]));
    // pressure gradient of the new h (agrid.py:55-69, barotr_pure.py:57-60)
    const T* pbx = s_hn + (a * RJ + (q + kHalo));
    const T* pby = s_hn + ((a + kHalo) * RJ + q);
    const T pgu = T(-9.80) * (rdx * (mid6(pbx + RJ, RJ) - mid6(pbx, RJ)));
    const T pgv = T(-9.80) * (rdy * (mid6(pby + 1, 1) - mid6(pby, 1)));
    const T af = s_af[e];
    // momentum update (barotr_pure.py:149-150)
    io.u_out[o] = s_up[e] + (pgu + advx + af * vct + visx) * io.dt;
    io.v_out[o] = s_vp[e] + (pgv + advy - af * uct + visy) * io.dt;
  }
}

// One tile phase with the prologue issued first (the stream/graph kernels).
template <typename T, int TI, int TJ>
__device__ __forceinline__ void tile_h(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm) {
  Gather<T, TI, TJ, false> gat;
  int cnt[4], P;
  tile_h_pro<T, TI, TJ>(g, io, b, sm, gat, cnt, P);
  wait_prior_grid();
  tile_h_main<T, TI, TJ>(g, io, b, sm, gat, cnt, P);
}
template <typename T, int TI, int TJ>
__device__ __forceinline__ void tile_uv(const Geo<T>& g, const StageIO<T>& io, const TileBox& b, T* sm) {
  Gather<T, TI, TJ, true> gat;
  int cnt[4], P;
  tile_uv_pro<T, TI, TJ>(g, io, b, sm, gat, cnt, P);
  wait_prior_grid();
  tile_uv_main<T, TI, TJ>(g, io, b, sm, gat, cnt, P);
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
  io.fx = a.fx;
  io.fy = a.fy;
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
