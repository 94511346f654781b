// bt_capi.cu - plan construction and the C-ABI of libbt.so (see include/licom_bt.h).

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "bt_plan.cuh"

using namespace bt;

namespace {
thread_local std::string g_err;
}  // namespace

namespace bt {
int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace bt

namespace {

int fail(int code, const std::string& msg) { return set_error(code, msg); }

int cuda_fail(cudaError_t e, const char* what) {
  return fail(BT_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BT_CUDA(call, what)                  \
  do {                                       \
    cudaError_t e_ = (call);                 \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

// Cube adjacency for side d of face t (0-based faces, sides E W N S = 0..3):
// even/odd face rules of the reference topology (communication.py:57-87); the
// along-edge index is reversed when an E/W side meets an S/N side
// (communication.py:41-55).
void face_neighbor(int t, int d, int* nb, int* side, int* rev) {
  if (t % 2 == 0) {
    switch (d) {
      case kS: *nb = (t + 4) % 6; *side = kE; break;
      case kE: *nb = (t + 2) % 6; *side = kS; break;
      case kN: *nb = (t + 1) % 6; *side = kS; break;
      default: *nb = (t + 5) % 6; *side = kE; break;
    }
  } else {
    switch (d) {
      case kE: *nb = (t + 1) % 6; *side = kW; break;
      case kN: *nb = (t + 2) % 6; *side = kW; break;
      case kW: *nb = (t + 4) % 6; *side = kN; break;
      default: *nb = (t + 5) % 6; *side = kN; break;
    }
  }
  const bool ew_a = (d == kE || d == kW), ew_b = (*side == kE || *side == kW);
  *rev = (ew_a != ew_b) ? 1 : 0;
}

// Interior cell on line c (0..2, in the order of communication.py:193-207)
// and along-edge position k next to ``side``.
void side_line_cell(int side, int c, int k, int m, int* i, int* j) {
  switch (side) {
    case kE: *i = kHalo + k; *j = m - 6 + c; break;
    case kW: *i = kHalo + k; *j = kHalo + c; break;
    case kN: *i = m - 6 + c; *j = kHalo + k; break;
    default: *i = kHalo + c; *j = kHalo + k; break;
  }
}

// Halo cell written from line c at position k of the band on side d
// (communication.py:210-223 without corners).
void band_cell(int d, int c, int k, int m, int* i, int* j) {
  switch (d) {
    case kE: *i = kHalo + k; *j = m - kHalo + c; break;
    case kW: *i = kHalo + k; *j = c; break;
    case kN: *i = m - kHalo + c; *j = kHalo + k; break;
    default: *i = c; *j = kHalo + k; break;
  }
}

}  // namespace

namespace {

// Halo gather tables of one resolution, host side: for every halo cell of
// every face, the two neighbour-interior source cells and the two linear
// interpolation weights (composition of communication.py:387-474 and
// cube.py:40-127); route[f*4+side] packs the adjacency.
template <typename T>
int build_halo_host(int n, const T* coef, const int* li, const int* lj, int2* src, T* w, int* route) {
  const int m = n + 6, nh = halo_count(m);
  const size_t fe = (size_t)6 * m * m;
  for (int f = 0; f < 6; ++f)
    for (int dd = 0; dd < 4; ++dd) {
      int nb, side, rev;
      face_neighbor(f, dd, &nb, &side, &rev);
      route[f * 4 + dd] = route_pack(nb, side, rev);
    }
  // halo copy map: halo band cell -> neighbour interior cell
  std::vector<long> copy(fe, -1);
  for (int f = 0; f < 6; ++f)
    for (int dd = 0; dd < 4; ++dd) {
      int nb, side, rev;
      face_neighbor(f, dd, &nb, &side, &rev);
      for (int c = 0; c < kHalo; ++c)
        for (int k = 0; k < n; ++k) {
          const int kk = rev ? n - 1 - k : k;
          int si, sj, ti, tj;
          side_line_cell(side, c, kk, m, &si, &sj);
          band_cell(dd, c, k, m, &ti, &tj);
          copy[cell(f, ti, tj, m)] = cell(nb, si, sj, m);
        }
    }
  // kinked->extended interpolation along the band; corners copy the band cell
  // of row 3 / M-4 (cube.py:64-125)
  for (int f = 0; f < 6; ++f)
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        if (is_interior(i, j, m)) continue;
        int bi = i;
        const int bj = j;
        const bool corner = (i < kHalo || i >= m - kHalo) && (j < kHalo || j >= m - kHalo);
        if (corner) bi = (i < kHalo) ? kHalo : m - kHalo - 1;
        const long ob = cell(f, bi, bj, m);
        const bool along_i = (bj < kHalo || bj >= m - kHalo);  // W/E band: interpolate along axis -2
        const int loc = along_i ? li[ob] : lj[ob];
        if (loc < kHalo || loc > m - kHalo - 2)
          return fail(BT_EINVAL, "k2e location table out of range at a halo cell (face " + std::to_string(f) +
                                     ", " + std::to_string(bi) + ", " + std::to_string(bj) + ")");
        long s0, s1;
        if (along_i) {
          s0 = copy[cell(f, loc, bj, m)];
          s1 = copy[cell(f, loc + 1, bj, m)];
        } else {
          s0 = copy[cell(f, bi, loc, m)];
          s1 = copy[cell(f, bi, loc + 1, m)];
        }
        if (s0 < 0 || s1 < 0) return fail(BT_EINVAL, "halo gather source is not a band cell");
        const size_t k = (size_t)f * nh + halo_id(i, j, m);
        src[k] = make_int2((int)s0, (int)s1);
        w[2 * k] = coef[2 * ob];
        w[2 * k + 1] = coef[2 * ob + 1];
      }
  return BT_OK;
}

template <typename T>
int build_tables(bt_plan* p, const bt_grid_desc* d) {
  const int m = p->m, nh = p->nh;
  const size_t fe = (size_t)6 * m * m;
  std::vector<T> coef(fe * 2), inner(fe), outer(fe);
  std::vector<int> li(fe), lj(fe);
  BT_CUDA(cudaMemcpy(coef.data(), d->k2e_coef, coef.size() * sizeof(T), cudaMemcpyDeviceToHost), "copy k2e_coef");
  BT_CUDA(cudaMemcpy(li.data(), d->loc_i_local, li.size() * sizeof(int), cudaMemcpyDeviceToHost), "copy loc_i");
  BT_CUDA(cudaMemcpy(lj.data(), d->loc_j_local, lj.size() * sizeof(int), cudaMemcpyDeviceToHost), "copy loc_j");
  BT_CUDA(cudaMemcpy(inner.data(), d->inner, fe * sizeof(T), cudaMemcpyDeviceToHost), "copy inner");
  BT_CUDA(cudaMemcpy(outer.data(), d->outer, fe * sizeof(T), cudaMemcpyDeviceToHost), "copy outer");
  // The kernels apply the ext_vector masks as exact 1/0 (cube.py:139-151): check them.
  for (int f = 0; f < 6; ++f)
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        const long o = cell(f, i, j, m);
        const T want = is_interior(i, j, m) ? T(1) : T(0);
        if (inner[o] != want || outer[o] != T(1) - want)
          return fail(BT_ENOTSUP, "inner/outer must be the interior/halo masks of duogrid.py:159-190");
      }
  std::vector<int2> src((size_t)6 * nh);
  std::vector<T> w((size_t)6 * nh * 2);
  const int rc = build_halo_host<T>(p->n, coef.data(), li.data(), lj.data(), src.data(), w.data(), p->route);
  if (rc != BT_OK) return rc;
  p->h_src = src;
  BT_CUDA(cudaMalloc(&p->d_hsrc, src.size() * sizeof(int2)), "alloc halo table");
  BT_CUDA(cudaMalloc(&p->d_hw, w.size() * sizeof(T)), "alloc halo weights");
  BT_CUDA(cudaMemcpy(p->d_hsrc, src.data(), src.size() * sizeof(int2), cudaMemcpyHostToDevice), "upload table");
  BT_CUDA(cudaMemcpy(p->d_hw, w.data(), w.size() * sizeof(T), cudaMemcpyHostToDevice), "upload weights");
  return BT_OK;
}

template <typename T>
StageIO<T> stage_io(const bt_plan* p, const T* h, const T* u, const T* v, const T* hp, const T* up, const T* vp,
                    T* ho, T* uo, T* vo, double dt, double beta, int stored, int last) {
  StageIO<T> io;
  io.fx = (T*)p->face_x();
  io.h = h;
  io.u = u;
  io.v = v;
  io.hp = hp;
  io.up = up;
  io.vp = vp;
  io.h_out = ho;
  io.u_out = uo;
  io.v_out = vo;
  io.dt = (T)dt;
  io.beta = (T)beta;
  io.stored_halo = stored;
  io.last = last;
  return io;
}

template <typename T>
cudaError_t run_stage(const bt_plan* p, const Geo<T>& g, const StageIO<T>& io, cudaStream_t s) {
  cudaEvent_t stop;
  cudaError_t e = p->time_begin(BT_KERNEL_PHASE_H, s, &stop);
  if (e == cudaSuccess) e = launch_phase_h<T>(g, io, p->tile, s, p->full_tiles);
  if (e == cudaSuccess && stop) e = cudaEventRecord(stop, s);
  if (e == cudaSuccess) e = p->time_begin(BT_KERNEL_PHASE_UV, s, &stop);
  if (e == cudaSuccess) e = launch_phase_uv<T>(g, io, p->tile, s, p->full_tiles);
  if (e == cudaSuccess && stop) e = cudaEventRecord(stop, s);
  return e;
}

// The launch sequence of one round (stream order).
template <typename T>
cudaError_t enqueue_round(const bt_plan* p, const bt_state_in& in, const bt_state_out& out, int nbb,
                          double dtb, int rk, cudaStream_t s) {
  const Geo<T> g = p->geo<T>();
  T* Y[3] = {(T*)p->scratch_field(0), (T*)p->scratch_field(1), (T*)p->scratch_field(2)};
  T* Z[3] = {(T*)p->scratch_field(3), (T*)p->scratch_field(4), (T*)p->scratch_field(5)};
  T* X[3] = {(T*)out.h0, (T*)out.ub, (T*)out.vb};
  const T* X0[3] = {(const T*)in.h0, (const T*)in.ub, (const T*)in.vb};
  const T* B0[3] = {(const T*)in.h0p, (const T*)in.ubp, (const T*)in.vbp};
  cudaError_t e = cudaSuccess;
  for (int step = 0; step < nbb; ++step) {
    const T* const* cur = step == 0 ? X0 : (const T* const*)X;
    const T* const* base = step == 0 ? B0 : (const T* const*)X;
    const int stored = step == 0 ? 1 : 0;
    if (rk == 2) {
      // barotr.py:50-56: dt/2 from the base, then dt from the same base
      e = run_stage<T>(p, g, stage_io<T>(p, cur[0], cur[1], cur[2], base[0], base[1], base[2], Y[0], Y[1], Y[2],
                                         dtb / 2.0, 0.0, stored, 0), s);
      if (e != cudaSuccess) return e;
      e = run_stage<T>(p, g, stage_io<T>(p, Y[0], Y[1], Y[2], base[0], base[1], base[2], X[0], X[1], X[2], dtb,
                                         0.0, 0, 1), s);
    } else {
      // barotr.py:73-83: dt/3, dt/2, dt with beta_d = 1
      e = run_stage<T>(p, g, stage_io<T>(p, cur[0], cur[1], cur[2], base[0], base[1], base[2], Y[0], Y[1], Y[2],
                                         dtb / 3.0, 1.0, stored, 0), s);
      if (e != cudaSuccess) return e;
      e = run_stage<T>(p, g, stage_io<T>(p, Y[0], Y[1], Y[2], base[0], base[1], base[2], Z[0], Z[1], Z[2],
                                         dtb / 2.0, 1.0, 0, 0), s);
      if (e != cudaSuccess) return e;
      e = run_stage<T>(p, g, stage_io<T>(p, Z[0], Z[1], Z[2], base[0], base[1], base[2], X[0], X[1], X[2], dtb,
                                         1.0, 0, 1), s);
    }
    if (e != cudaSuccess) return e;
  }
  if (out.diag[0]) {
    T* const* L = rk == 2 ? Y : Z;  // input of the last stage
    e = launch_fill_halo<T>(g, L[0], L[1], L[2], s);
    if (e != cudaSuccess) return e;
    DiagOut<T> d;
    T** dp = (T**)&d;
    for (int k = 0; k < 10; ++k) dp[k] = (T*)out.diag[k];
    e = launch_diag<T>(g, L[0], L[1], L[2], d, s);
    if (e != cudaSuccess) return e;
  }
  return launch_fill_halo<T>(g, X[0], X[1], X[2], s);
}

template <typename T>
cudaError_t enqueue_stage(const bt_plan* p, const bt_state_in& in, const bt_state_out& out, double dt,
                          double beta, int last, cudaStream_t s) {
  const Geo<T> g = p->geo<T>();
  T* X[3] = {(T*)out.h0, (T*)out.ub, (T*)out.vb};
  const StageIO<T> io = stage_io<T>(p, (const T*)in.h0, (const T*)in.ub, (const T*)in.vb, (const T*)in.h0p,
                                    (const T*)in.ubp, (const T*)in.vbp, X[0], X[1], X[2], dt, beta, 1, last);
  cudaError_t e = run_stage<T>(p, g, io, s);
  if (e != cudaSuccess) return e;
  if (out.diag[0]) {
    DiagOut<T> d;
    T** dp = (T**)&d;
    for (int k = 0; k < 10; ++k) dp[k] = (T*)out.diag[k];
    e = launch_diag<T>(g, (const T*)in.h0, (const T*)in.ub, (const T*)in.vb, d, s);
    if (e != cudaSuccess) return e;
  }
  return launch_fill_halo<T>(g, X[0], X[1], X[2], s);
}

}  // namespace

namespace bt {
// Tile constant blocks of plan p for tile shape t (Geo::cblk): built once per
// shape into a buffer of their own on stream s, which is then synchronised, so
// rounds on any stream may use them afterwards; without them (allocation
// failure) the phases read the constant arrays as before.  Runs before any
// capture of the round (bt_round builds them ahead of its graph), so the
// first round of a plan per tile shape must not be inside a stream capture.
template <typename T>
int ensure_const_blocks(bt_plan* p, TileCfg t, cudaStream_t s) {
  if (p->cblk_for(t)) return BT_OK;
  const size_t bytes = const_block_elems(t, p->n) * sizeof(T);
  bt_plan::ConstBlocks* slot = nullptr;
  for (bt_plan::ConstBlocks& c : p->cblks)
    if (!c.ptr) slot = &c;
  if (bytes == 0 || !slot) return BT_OK;
  if (cudaMalloc(&slot->ptr, bytes) != cudaSuccess) {
    cudaGetLastError();  // clear the allocation error: the arrays serve instead
    slot->ptr = nullptr;
    return BT_OK;
  }
  cudaError_t e = launch_const_blocks<T>(p->geo_arrays<T>(), t, (T*)slot->ptr, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaFree(slot->ptr);
    slot->ptr = nullptr;
    return set_error(BT_ECUDA, std::string("tile constant blocks: ") + cudaGetErrorString(e));
  }
  slot->tile = t;
  return BT_OK;
}

int ensure_const_blocks_any(bt_plan* p, TileCfg t, cudaStream_t s) {
  return p->dtype == BT_F64 ? ensure_const_blocks<double>(p, t, s) : ensure_const_blocks<float>(p, t, s);
}
}  // namespace bt

namespace {

// Substeps per cooperative launch of the persistent and resident modes: a
// round is split into launches of at most this many substeps, so the grid
// barrier's 31-bit arrival count (2 x stages x substeps x CTAs) and the
// resident progress flags (2 x stages x substeps) stay far from overflow.
constexpr int kSubstepsPerLaunch = 1 << 16;

// The launch arguments of a whole round (persistent and resident modes).
template <typename T>
RoundArgs<T> round_args(bt_plan* p, const bt_state_in& in, const bt_state_out& out, int nbb, double dtb,
                        int rk) {
  RoundArgs<T> a;
  a.g = p->geo<T>();
  for (int k = 0; k < 3; ++k) {
    a.y[k] = (T*)p->scratch_field(k);
    a.z[k] = (T*)p->scratch_field(3 + k);
  }
  a.x0[0] = (const T*)in.h0;
  a.x0[1] = (const T*)in.ub;
  a.x0[2] = (const T*)in.vb;
  a.b0[0] = (const T*)in.h0p;
  a.b0[1] = (const T*)in.ubp;
  a.b0[2] = (const T*)in.vbp;
  a.x[0] = (T*)out.h0;
  a.x[1] = (T*)out.ub;
  a.x[2] = (T*)out.vb;
  a.fx = (T*)p->face_x();
  a.nbb = nbb;
  a.rk = rk;
  a.step0 = 0;
  a.dtb = dtb;
  a.bar = p->d_flags;
  a.err = (int*)(p->d_flags + 1);
  a.spin_limit = p->spin_limit;
  return a;
}

// Halo fill of the result and the diagnostics of the last stage after a
// persistent or resident round.
template <typename T>
cudaError_t round_epilogue(const RoundArgs<T>& a, const bt_state_out& out, int rk, cudaStream_t s) {
  cudaError_t e;
  const Geo<T>& g = a.g;
  if (out.diag[0]) {
    T* const* L = rk == 2 ? a.y : a.z;
    if ((e = launch_fill_halo<T>(g, L[0], L[1], L[2], s)) != cudaSuccess) return e;
    DiagOut<T> d;
    T** dp = (T**)&d;
    for (int k = 0; k < 10; ++k) dp[k] = (T*)out.diag[k];
    if ((e = launch_diag<T>(g, L[0], L[1], L[2], d, s)) != cudaSuccess) return e;
  }
  return launch_fill_halo<T>(g, a.x[0], a.x[1], a.x[2], s);
}

// Dependency lists of the resident kernel for tile shape c (see
// bt_resident.cuh): for every tile, the tiles owning a cell it reads in
// either phase of a stage -- the rectangle of 3 cells around the tile (halo
// cells resolved to their two gather sources) and, along the face edges the
// tile touches, the neighbour face's 6-point lines normal to the edge (their
// halo points resolved likewise) -- made symmetric, without the tile itself.
int build_resident_deps(bt_plan* p, TileCfg c) {
  if (p->res_tile.ti == c.ti && p->res_tile.tj == c.tj && p->d_res) return BT_OK;
  const int n = p->n, m = p->m, nh = p->nh;
  const Tiling t = make_tiling(c, n);
  const int ntiles = 6 * t.tiles_per_face();
  auto owner = [&](long o) {
    const int f = (int)(o / ((long)m * m));
    const int r = (int)(o - (long)f * m * m), i = r / m, j = r % m;
    return (f * t.nti + (i - kHalo) / t.ti) * t.ntj + (j - kHalo) / t.tj;
  };
  std::vector<std::vector<int>> dep(ntiles);
  auto add = [&](int tile, int f, int i, int j) {
    if (is_interior(i, j, m)) {
      dep[tile].push_back(owner(cell(f, i, j, m)));
    } else {
      const int2 sx = p->h_src[(size_t)f * nh + halo_id(i, j, m)];
      dep[tile].push_back(owner(sx.x));
      dep[tile].push_back(owner(sx.y));
    }
  };
  for (int f = 0; f < 6; ++f)
    for (int ti = 0; ti < t.nti; ++ti)
      for (int tj = 0; tj < t.ntj; ++tj) {
        const int tile = (f * t.nti + ti) * t.ntj + tj;
        const int i0 = kHalo + ti * t.ti, j0 = kHalo + tj * t.tj;
        const int ni = std::min(t.ti, n - ti * t.ti), nj = std::min(t.tj, n - tj * t.tj);
        for (int i = i0 - kHalo; i < i0 + ni + kHalo; ++i)
          for (int j = j0 - kHalo; j < j0 + nj + kHalo; ++j) add(tile, f, i, j);
        const bool touch[4] = {j0 + nj == m - kHalo, j0 == kHalo, i0 + ni == m - kHalo, i0 == kHalo};  // E W N S
        for (int side = 0; side < 4; ++side) {
          if (!touch[side]) continue;
          const int r = p->route[f * 4 + side], nb = route_nb(r), ns = route_side(r);
          const bool along_j = side == kS || side == kN;
          const int k0 = along_j ? j0 - kHalo : i0 - kHalo, nk = along_j ? nj : ni;
          for (int k = k0; k < k0 + nk; ++k) {
            const int kk = route_rev(r) ? n - 1 - k : k;
            for (int q = 0; q < 6; ++q) {
              int i, j;
              edge_point(ns, kk, q, m, i, j);
              add(tile, nb, i, j);
            }
          }
        }
      }
  for (int tile = 0; tile < ntiles; ++tile)
    for (int d : std::vector<int>(dep[tile]))
      if (d != tile) dep[d].push_back(tile);
  std::vector<int> off(ntiles + 1, 0), idx;
  for (int tile = 0; tile < ntiles; ++tile) {
    std::vector<int>& v = dep[tile];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    for (int d : v) {
      if (d < 0 || d >= ntiles) return fail(BT_EINVAL, "resident mode: dependency outside the tile set");
      if (d != tile) idx.push_back(d);
    }
    off[tile + 1] = (int)idx.size();
  }
  if (p->d_res) {
    cudaFree(p->d_res);
    p->d_res = nullptr;
  }
  // offsets, lists, up to one line of padding, then one line per tile's flag and one for the abort word
  const size_t words = (ntiles + 1) + idx.size() + kResFlagStride + (size_t)(ntiles + 1) * kResFlagStride;
  if (cudaMalloc(&p->d_res, words * sizeof(int)) != cudaSuccess)
    return fail(BT_ENOMEM, "resident mode: dependency table allocation failed");
  std::vector<int> blob(off);
  blob.insert(blob.end(), idx.begin(), idx.end());
  BT_CUDA(cudaMemcpy(p->d_res, blob.data(), blob.size() * sizeof(int), cudaMemcpyHostToDevice),
          "resident mode: upload dependency table");
  p->res_tile = c;
  p->res_tiles = ntiles;
  p->res_ndep = (int)idx.size();
  return BT_OK;
}

// Resident mode: one cooperative launch with one CTA per tile runs every
// phase of every substep (bt_resident.cuh); the plan's tile shape must be a
// resident shape whose tiles all fit on the device at once.
template <typename T>
int enqueue_round_resident(bt_plan* p, const bt_state_in& in, const bt_state_out& out, int nbb, double dtb,
                           int rk, cudaStream_t s) {
  if (!resident_tile_supported(p->tile))
    return fail(BT_ENOTSUP, "bt_round: resident mode supports the tile shapes 8x16, 16x16 and 8x32");
  int cap = 0;
  cudaError_t e = resident_capacity<T>(p->tile, &cap);
  if (e != cudaSuccess) return cuda_fail(e, "bt_round: resident occupancy");
  const int ntiles = 6 * make_tiling(p->tile, p->n).tiles_per_face();
  if (ntiles > cap)
    return fail(BT_ENOTSUP, "bt_round: resident mode needs all " + std::to_string(ntiles) +
                                " tiles on the GPU at once, " + std::to_string(cap) +
                                " fit: use a larger tile or graph mode");
  const int rc = build_resident_deps(p, p->tile);
  if (rc != BT_OK) return rc;
  RoundArgs<T> a = round_args<T>(p, in, out, nbb, dtb, rk);
  ResSync rs;
  rs.dep_off = p->d_res;
  rs.dep_idx = p->d_res + ntiles + 1;
  // flags start on a 128-byte boundary, one line per tile, the abort word on the line after them
  const size_t flag0 = ((size_t)ntiles + 1 + p->res_ndep + kResFlagStride - 1) / kResFlagStride * kResFlagStride;
  rs.flags = p->d_res + flag0;
  rs.abort = rs.flags + (size_t)ntiles * kResFlagStride;
  p->last_grid = ntiles;
  for (int step0 = 0; step0 < nbb; step0 += kSubstepsPerLaunch) {
    a.step0 = step0;
    a.nbb = std::min(kSubstepsPerLaunch, nbb - step0);
    if ((e = cudaMemsetAsync(rs.flags, 0, ((size_t)ntiles + 1) * kResFlagStride * sizeof(int), s)) != cudaSuccess)
      return cuda_fail(e, "bt_round: resident flags");
    cudaEvent_t t1 = nullptr;
    if ((e = p->time_begin(BT_KERNEL_ROUND, s, &t1)) != cudaSuccess) return cuda_fail(e, "bt_round: timing");
    if ((e = launch_resident<T>(a, rs, p->tile, s)) != cudaSuccess) return cuda_fail(e, "bt_round: resident launch");
    if (t1 && (e = cudaEventRecord(t1, s)) != cudaSuccess) return cuda_fail(e, "bt_round: timing");
  }
  if ((e = round_epilogue<T>(a, out, rk, s)) != cudaSuccess) return cuda_fail(e, "bt_round: halo fill");
  return BT_OK;
}

// Persistent mode: one cooperative launch runs every phase of every substep.
template <typename T>
cudaError_t enqueue_round_persistent(bt_plan* p, const bt_state_in& in, const bt_state_out& out, int nbb,
                                     double dtb, int rk, cudaStream_t s) {
  RoundArgs<T> a = round_args<T>(p, in, out, nbb, dtb, rk);
  for (int step0 = 0; step0 < nbb; step0 += kSubstepsPerLaunch) {
    a.step0 = step0;
    a.nbb = std::min(kSubstepsPerLaunch, nbb - step0);
    cudaError_t e = cudaMemsetAsync(p->d_flags, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    cudaEvent_t t1 = nullptr;
    if ((e = p->time_begin(BT_KERNEL_ROUND, s, &t1)) != cudaSuccess) return e;
    e = launch_round<T>(a, p->tile, p->max_ctas, s, &p->last_grid);
    if (e != cudaSuccess) return e;
    if (t1 && (e = cudaEventRecord(t1, s)) != cudaSuccess) return e;
  }
  return round_epilogue<T>(a, out, rk, s);
}

cudaError_t enqueue(const bt_plan* p, const bt_state_in& in, const bt_state_out& out, int nbb, double dtb,
                    int rk, cudaStream_t s) {
  return p->dtype == BT_F64 ? enqueue_round<double>(p, in, out, nbb, dtb, rk, s)
                            : enqueue_round<float>(p, in, out, nbb, dtb, rk, s);
}

// ---- edge average kernels (bt_edge_average) --------------------------------
template <typename T>
__global__ void k_edge_gather(Geo<T> g, const T* u, const T* v, T* lines) {
  const int n = g.n, m = g.m;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 24 * n) return;
  const int fd = k / n, q = k - fd * n, f = fd / 4, d = fd % 4;
  long o;
  const T* src;
  switch (d) {
    case kE: o = cell(f, kHalo + q, m - kHalo, m); src = v; break;
    case kW: o = cell(f, kHalo + q, kHalo, m); src = v; break;
    case kN: o = cell(f, m - kHalo, kHalo + q, m); src = u; break;
    default: o = cell(f, kHalo, kHalo + q, m); src = u; break;
  }
  lines[k] = src[o];
}

template <typename T>
__global__ void k_edge_apply(Geo<T> g, T* u, T* v, const T* lines) {
  const int n = g.n, m = g.m;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 24 * n) return;
  const int fd = k / n, q = k - fd * n, f = fd / 4, d = fd % 4;
  const int r = g.route[fd];
  const int kk = route_rev(r) ? n - 1 - q : q;
  const T val = (lines[k] + lines[(route_nb(r) * 4 + route_side(r)) * n + kk]) / T(2.0);
  switch (d) {
    case kE: v[cell(f, kHalo + q, m - kHalo, m)] = val; break;
    case kW: v[cell(f, kHalo + q, kHalo, m)] = val; break;
    case kN: u[cell(f, m - kHalo, kHalo + q, m)] = val; break;
    default: u[cell(f, kHalo, kHalo + q, m)] = val; break;
  }
}

template <typename T>
cudaError_t enqueue_edge_average(const bt_plan* p, void* u, void* v, cudaStream_t s) {
  const Geo<T> g = p->geo<T>();
  const int total = 24 * p->n, th = 128, bl = (total + th - 1) / th;
  k_edge_gather<T><<<bl, th, 0, s>>>(g, (const T*)u, (const T*)v, (T*)p->edge_lines());
  k_edge_apply<T><<<bl, th, 0, s>>>(g, (T*)u, (T*)v, (const T*)p->edge_lines());
  return cudaGetLastError();
}

}  // namespace

extern "C" {

int bt_version(void) { return 1; }

int bt_halo_table_host(int n, const double* k2e_coef, const int* loc_i, const int* loc_j, int* src,
                       double* weights, int* route) {
  if (n < 4 || !k2e_coef || !loc_i || !loc_j || !src || !weights || !route)
    return fail(BT_EINVAL, "bt_halo_table_host: bad argument");
  return build_halo_host<double>(n, k2e_coef, loc_i, loc_j, (int2*)src, weights, route);
}

const char* bt_last_error(void) { return g_err.c_str(); }

int bt_plan_create(const bt_grid_desc* d, bt_plan** out) {
  if (!d || !out) return fail(BT_EINVAL, "bt_plan_create: NULL argument");
  *out = nullptr;
  if (d->n < 4 || d->n > 8192) return fail(BT_EINVAL, "bt_plan_create: n must be in [4, 8192]");
  if (d->dtype != BT_F64 && d->dtype != BT_F32) return fail(BT_EINVAL, "bt_plan_create: dtype must be BT_F64 or BT_F32");
  const void* cs[17] = {d->dzph_x, d->dzph_y, d->rdx, d->rdy, d->a_f, d->k2e_coef, d->loc_i_local,
                        d->loc_j_local, d->a_c2l, d->a_l2c, d->inner, d->outer, d->a_gct, d->a_sina,
                        d->rda, d->c_dy, d->d_dx};
  for (int k = 0; k < 17; ++k)
    if (!cs[k]) return fail(BT_EINVAL, "bt_plan_create: constant pointer " + std::to_string(k) + " is NULL");
  if (!matrices_aligned(d)) return fail(BT_EINVAL, "bt_plan_create: a_c2l, a_l2c and a_gct must be 16-byte aligned");
  bt_plan* p = new bt_plan;
  p->n = d->n;
  p->m = d->n + 6;
  p->nh = halo_count(p->m);
  p->dtype = d->dtype;
  std::memcpy(p->c, cs, sizeof(cs));
  cudaGetDevice(&p->device);
  p->field_elems = (size_t)6 * p->m * p->m;
  cudaError_t pe = p->dtype == BT_F64 ? prime_kernels<double>() : prime_kernels<float>();
  if (pe == cudaSuccess) pe = p->dtype == BT_F64 ? prime_resident<double>() : prime_resident<float>();
  if (pe != cudaSuccess) {
    bt_plan_destroy(p);
    return cuda_fail(pe, "bt_plan_create: kernel attributes");
  }
  int rc = p->dtype == BT_F64 ? build_tables<double>(p, d) : build_tables<float>(p, d);
  if (rc != BT_OK) {
    bt_plan_destroy(p);
    return rc;
  }
  const size_t bytes = p->scratch_bytes();
  cudaError_t e = cudaMalloc(&p->scratch, bytes);
  if (e != cudaSuccess) {
    bt_plan_destroy(p);
    return fail(BT_ENOMEM, std::string("bt_plan_create: scratch allocation: ") + cudaGetErrorString(e));
  }
  e = cudaMalloc(&p->d_flags, 2 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(p->d_flags, 0, 2 * sizeof(unsigned));
  if (e != cudaSuccess) {
    bt_plan_destroy(p);
    return fail(BT_ENOMEM, std::string("bt_plan_create: flag allocation: ") + cudaGetErrorString(e));
  }
  e = cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    bt_plan_destroy(p);
    return cuda_fail(e, "bt_plan_create: stream/event");
  }
  *out = p;
  return BT_OK;
}

int bt_plan_destroy(bt_plan* p) {
  if (!p) return BT_OK;
  if (p->gexec) cudaGraphExecDestroy(p->gexec);
  if (p->ev_in) cudaEventDestroy(p->ev_in);
  if (p->ev_out) cudaEventDestroy(p->ev_out);
  for (cudaEvent_t ev : p->tev) cudaEventDestroy(ev);
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
  if (p->scratch) cudaFree(p->scratch);
  if (p->d_flags) cudaFree(p->d_flags);
  if (p->d_hsrc) cudaFree(p->d_hsrc);
  if (p->d_hw) cudaFree(p->d_hw);
  if (p->d_res) cudaFree(p->d_res);
  for (bt_plan::ConstBlocks& c : p->cblks)
    if (c.ptr) cudaFree(c.ptr);
  delete p;
  return BT_OK;
}

int bt_plan_set_tile(bt_plan* p, int ti, int tj) {
  if (!p) return fail(BT_EINVAL, "bt_plan_set_tile: NULL plan");
  if (!tile_cfg_supported({ti, tj})) return fail(BT_EINVAL, "bt_plan_set_tile: unsupported tile shape");
  p->tile = {ti, tj};
  if (p->gexec) {
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
    p->gkey.clear();
  }
  return BT_OK;
}

int bt_plan_set_mode(bt_plan* p, int mode) {
  if (!p) return fail(BT_EINVAL, "bt_plan_set_mode: NULL plan");
  if (mode != BT_MODE_STREAM && mode != BT_MODE_GRAPH && mode != BT_MODE_PERSISTENT && mode != BT_MODE_RESIDENT)
    return fail(BT_EINVAL, "bt_plan_set_mode: unknown mode");
  p->mode = mode;
  return BT_OK;
}

int bt_round(bt_plan* p, const bt_state_in* in, const bt_state_out* out, int nbb, double dtb, int rk,
             void* stream) {
  if (!p || !in || !out) return fail(BT_EINVAL, "bt_round: NULL argument");
  if (rk != 2 && rk != 3) return fail(BT_EINVAL, "bt_round: rk must be 2 or 3");
  if (nbb < 1) return fail(BT_EINVAL, "bt_round: nbb must be >= 1");
  const void* ins[6] = {in->h0, in->h0p, in->ub, in->vb, in->ubp, in->vbp};
  for (const void* q : ins)
    if (!q) return fail(BT_EINVAL, "bt_round: NULL input field");
  if (!out->h0 || !out->ub || !out->vb) return fail(BT_EINVAL, "bt_round: NULL output field");
  for (const void* q : ins)
    if (q == out->h0 || q == out->ub || q == out->vb)
      return fail(BT_EINVAL, "bt_round: output fields must not alias the inputs");
  if (out->diag[0])
    for (int k = 1; k < 10; ++k)
      if (!out->diag[k]) return fail(BT_EINVAL, "bt_round: diag outputs must be all set or diag[0] NULL");
  cudaStream_t s = (cudaStream_t)stream;
  {
    const int rc = ensure_const_blocks_any(p, p->tile, s);
    if (rc != BT_OK) return rc;
  }
  if (p->mode == BT_MODE_RESIDENT)
    return p->dtype == BT_F64 ? enqueue_round_resident<double>(p, *in, *out, nbb, dtb, rk, s)
                              : enqueue_round_resident<float>(p, *in, *out, nbb, dtb, rk, s);
  if (p->mode == BT_MODE_PERSISTENT) {
    cudaError_t e = p->dtype == BT_F64 ? enqueue_round_persistent<double>(p, *in, *out, nbb, dtb, rk, s)
                                       : enqueue_round_persistent<float>(p, *in, *out, nbb, dtb, rk, s);
    if (e != cudaSuccess) return cuda_fail(e, "bt_round: persistent launch");
    return BT_OK;
  }
  if (p->mode == BT_MODE_STREAM) {
    cudaError_t e = enqueue(p, *in, *out, nbb, dtb, rk, s);
    if (e != cudaSuccess) return cuda_fail(e, "bt_round: launch");
    return BT_OK;
  }
  // graph mode: capture once per (nbb, rk, dtb, pointers), replay afterwards
  std::vector<uintptr_t> key = {(uintptr_t)nbb, (uintptr_t)rk};
  uint64_t dbits;
  std::memcpy(&dbits, &dtb, 8);
  key.push_back((uintptr_t)dbits);
  for (const void* q : ins) key.push_back((uintptr_t)q);
  key.push_back((uintptr_t)out->h0);
  key.push_back((uintptr_t)out->ub);
  key.push_back((uintptr_t)out->vb);
  for (int k = 0; k < 10; ++k) key.push_back((uintptr_t)out->diag[k]);
  BT_CUDA(cudaEventRecord(p->ev_in, s), "bt_round: event record");
  BT_CUDA(cudaStreamWaitEvent(p->cap_stream, p->ev_in, 0), "bt_round: stream wait");
  if (!p->gexec || key != p->gkey) {
    if (p->gexec) {
      cudaGraphExecDestroy(p->gexec);
      p->gexec = nullptr;
    }
    cudaGraph_t graph;
    BT_CUDA(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal), "bt_round: begin capture");
    cudaError_t e = enqueue(p, *in, *out, nbb, dtb, rk, p->cap_stream);
    cudaError_t e2 = cudaStreamEndCapture(p->cap_stream, &graph);
    if (e != cudaSuccess) return cuda_fail(e, "bt_round: capture launch");
    if (e2 != cudaSuccess) return cuda_fail(e2, "bt_round: end capture");
    e = cudaGraphInstantiate(&p->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "bt_round: graph instantiate");
    p->gkey = key;
  }
  BT_CUDA(cudaGraphLaunch(p->gexec, p->cap_stream), "bt_round: graph launch");
  BT_CUDA(cudaEventRecord(p->ev_out, p->cap_stream), "bt_round: event record");
  BT_CUDA(cudaStreamWaitEvent(s, p->ev_out, 0), "bt_round: stream wait");
  return BT_OK;
}

int bt_stage(bt_plan* p, const bt_state_in* in, const bt_state_out* out, double dt, double beta_d,
             int is_laststep, void* stream) {
  if (!p || !in || !out) return fail(BT_EINVAL, "bt_stage: NULL argument");
  const void* ins[6] = {in->h0, in->h0p, in->ub, in->vb, in->ubp, in->vbp};
  for (const void* q : ins)
    if (!q) return fail(BT_EINVAL, "bt_stage: NULL input field");
  if (!out->h0 || !out->ub || !out->vb) return fail(BT_EINVAL, "bt_stage: NULL output field");
  for (const void* q : ins)
    if (q == out->h0 || q == out->ub || q == out->vb)
      return fail(BT_EINVAL, "bt_stage: output fields must not alias the inputs");
  if (out->diag[0])
    for (int k = 1; k < 10; ++k)
      if (!out->diag[k]) return fail(BT_EINVAL, "bt_stage: diag outputs must be all set or diag[0] NULL");
  cudaStream_t s = (cudaStream_t)stream;
  {
    const int rc = ensure_const_blocks_any(p, p->tile, s);
    if (rc != BT_OK) return rc;
  }
  cudaError_t e = p->dtype == BT_F64 ? enqueue_stage<double>(p, *in, *out, dt, beta_d, is_laststep ? 1 : 0, s)
                                     : enqueue_stage<float>(p, *in, *out, dt, beta_d, is_laststep ? 1 : 0, s);
  if (e != cudaSuccess) return cuda_fail(e, "bt_stage: launch");
  return BT_OK;
}

int bt_fill_halo(bt_plan* p, void* h, void* u, void* v, void* stream) {
  if (!p) return fail(BT_EINVAL, "bt_fill_halo: NULL plan");
  if ((u == nullptr) != (v == nullptr)) return fail(BT_EINVAL, "bt_fill_halo: u and v must both be set or NULL");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = p->dtype == BT_F64
                      ? launch_fill_halo<double>(p->geo<double>(), (double*)h, (double*)u, (double*)v, s)
                      : launch_fill_halo<float>(p->geo<float>(), (float*)h, (float*)u, (float*)v, s);
  if (e != cudaSuccess) return cuda_fail(e, "bt_fill_halo");
  return BT_OK;
}

int bt_edge_average(bt_plan* p, void* u, void* v, void* stream) {
  if (!p || !u || !v) return fail(BT_EINVAL, "bt_edge_average: NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = p->dtype == BT_F64 ? enqueue_edge_average<double>(p, u, v, s)
                                     : enqueue_edge_average<float>(p, u, v, s);
  if (e != cudaSuccess) return cuda_fail(e, "bt_edge_average");
  return BT_OK;
}

int bt_check_device_error(bt_plan* p) {
  if (!p) return fail(BT_EINVAL, "bt_check_device_error: NULL plan");
  BT_CUDA(cudaDeviceSynchronize(), "bt_check_device_error: synchronize");
  unsigned flags[2];
  BT_CUDA(cudaMemcpy(flags, p->d_flags, sizeof(flags), cudaMemcpyDeviceToHost), "bt_check_device_error: read flag");
  if (flags[1] != 0) {
    BT_CUDA(cudaMemset(p->d_flags + 1, 0, sizeof(unsigned)), "bt_check_device_error: clear flag");
    if (flags[1] & kErrBarrierTimeout)
      return fail(BT_EDEVICE, "persistent round: grid barrier wait exceeded its poll limit; the round was abandoned");
    if (flags[1] & kErrNeighbourTimeout)
      return fail(BT_EDEVICE, "resident round: a neighbour-tile wait exceeded its poll limit; the round was abandoned");
    return fail(BT_EDEVICE, "device error flag " + std::to_string(flags[1]));
  }
  return BT_OK;
}

int bt_plan_set_option(bt_plan* p, int key, long long value) {
  if (!p) return fail(BT_EINVAL, "bt_plan_set_option: NULL plan");
  switch (key) {
    case BT_OPT_MAX_CTAS:
      if (value < 0 || value > (1 << 20)) return fail(BT_EINVAL, "bt_plan_set_option: max_ctas out of range");
      p->max_ctas = (int)value;
      return BT_OK;
    case BT_OPT_SPIN_LIMIT:
      if (value < -1) return fail(BT_EINVAL, "bt_plan_set_option: spin limit must be >= -1");
      p->spin_limit = value;
      return BT_OK;
    case BT_OPT_KERNEL_TIMING:
      p->timing = value ? 1 : 0;
      p->tev_used = 0;
      return BT_OK;
    case BT_OPT_FULL_TILES:
      if (value < -1 || value > 1) return fail(BT_EINVAL, "bt_plan_set_option: full_tiles must be -1, 0 or 1");
      p->full_tiles = (int)value;
      if (p->gexec) {  // the captured round holds the previous kernels
        cudaGraphExecDestroy(p->gexec);
        p->gexec = nullptr;
        p->gkey.clear();
      }
      return BT_OK;
    default:
      return fail(BT_EINVAL, "bt_plan_set_option: unknown option");
  }
}

int bt_plan_kernel_time(bt_plan* p, int kind, double* ms_total, int* launches) {
  if (!p || !ms_total || !launches) return fail(BT_EINVAL, "bt_plan_kernel_time: NULL argument");
  double total = 0.0;
  int count = 0;
  for (size_t k = 0; k + 1 < p->tev_used; k += 2) {
    if (p->tkind[k / 2] != kind) continue;
    BT_CUDA(cudaEventSynchronize(p->tev[k + 1]), "bt_plan_kernel_time: synchronize");
    float ms = 0.f;
    BT_CUDA(cudaEventElapsedTime(&ms, p->tev[k], p->tev[k + 1]), "bt_plan_kernel_time: elapsed");
    total += ms;
    ++count;
  }
  *ms_total = total;
  *launches = count;
  return BT_OK;
}

long long bt_plan_get_info(bt_plan* p, int key) {
  if (!p) return -1;
  switch (key) {
    case BT_INFO_LAST_GRID: return p->last_grid;
    case BT_INFO_SCRATCH_BYTES: return (long long)p->scratch_bytes();
    case BT_INFO_FULL_TILES: {  // evaluated on the plan's device, as its launches are
      int cur = -1;
      cudaGetDevice(&cur);
      if (cur != p->device) cudaSetDevice(p->device);
      const int r = p->dtype == BT_F64 ? phase_full_paths<double>(p->tile, p->n, p->full_tiles)
                                       : phase_full_paths<float>(p->tile, p->n, p->full_tiles);
      if (cur >= 0 && cur != p->device) cudaSetDevice(cur);
      return r;
    }
    default: return -1;
  }
}

}  // extern "C"
