// bt_noalloc.cu - bt_round_noalloc: a round of the barotropic solver that allocates nothing.
//
// Some callers cannot allocate device memory: a custom-call handler of another
// framework's runtime that is handed only its operand buffers (the runtime owns
// the device memory pool), a Fortran or C model driver that reserves all of its
// GPU memory up front, or a service that must not change its memory footprint
// once it is serving.  bt_round does allocate (its plan owns stage scratch,
// face caches and the halo gather tables), so this file offers one entry point
// that keeps all of that scratch in a fixed array of device memory that the
// library declares statically.
//
// The array (kScratchBytes, 6 MiB) belongs to every GPU that loads the library
// and stays allocated until the process exits.  It holds, in this order: a
// status word, the halo gather tables, the stage fields (3, or 6 for RK3) and
// the face cache blocks of the 8 x 16 tiles.  The largest sizes that fit: float64 N <= 112 (RK2) /
// 96 (RK3), float32 N <= 160 (RK2) / 136 (RK3); larger sizes are rejected with
// BT_EINVAL.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress and sets the kernels'
// shared-memory limits; make that first call before any stream capture.
//
// Validation: the first call with a given set of constant pointers (per
// device) checks on the device what bt_plan_create checks on the host -- every
// k2e location the halo remap reads lies inside the band, and inner/outer are
// the exact interior / halo masks -- and waits for the answer (a stream
// synchronisation); tables that fail return BT_EINVAL / BT_ENOTSUP like
// bt_plan_create.  Later calls with the same pointers skip the check, so the
// tables must not change while they are in use (as for a plan).
//
// Every call reuses the same array and keeps whatever the previous call left
// there: the status word is cleared before each check; nothing else has to
// start at zero (the tables are rebuilt and every cache entry is written
// before it is read), but two calls whose work overlaps on the GPU (different
// streams, or one device used from several threads) race on it -- serialise
// them.
//
// Tile shape: the round runs the 8 x 16 tiles, the shape with the most CTAs
// at the sizes this entry point accepts (one full wave of 432 CTAs at N = 96,
// three per SM) and the one the autotuner picks for float64 at N = 96; the
// results are bitwise the same for every tile shape in float64.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "bt_launch.cuh"
#include "bt_plan.cuh"
#include "licom_bt.h"

namespace bt {
namespace {

constexpr size_t kScratchBytes = 6u << 20;  // 6 MiB
constexpr size_t kStatusBytes = 256;          // status word of the table check, then the scratch proper
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};
bool g_primed_f64[kMaxDevices] = {};
bool g_primed_f32[kMaxDevices] = {};

// The constant set last validated on each device (pointers, N, dtype).
struct CheckedDesc {
  bool valid = false;
  int n = 0, dtype = 0;
  const void* c[17] = {};
};
CheckedDesc g_checked[kMaxDevices];

enum NoallocStatus : unsigned { kBadLocation = 1u, kBadMask = 2u };

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Adjacency of the cube faces (the same rules as the plan's tables).
struct RouteTable {
  int r[24];
};

RouteTable make_routes() {
  RouteTable t;
  for (int f = 0; f < 6; ++f)
    for (int d = 0; d < 4; ++d) {
      int nb, side;
      if (f % 2 == 0) {
        switch (d) {
          case kS: nb = (f + 4) % 6; side = kE; break;
          case kE: nb = (f + 2) % 6; side = kS; break;
          case kN: nb = (f + 1) % 6; side = kS; break;
          default: nb = (f + 5) % 6; side = kE; break;
        }
      } else {
        switch (d) {
          case kE: nb = (f + 1) % 6; side = kW; break;
          case kN: nb = (f + 2) % 6; side = kW; break;
          case kW: nb = (f + 4) % 6; side = kN; break;
          default: nb = (f + 5) % 6; side = kN; break;
        }
      }
      const bool ew_a = (d == kE || d == kW), ew_b = (side == kE || side == kW);
      t.r[f * 4 + d] = route_pack(nb, side, ew_a != ew_b ? 1 : 0);
    }
  return t;
}

// Interior cell of the neighbouring face that the halo band cell (ti, tj) of
// face f copies (the halo copy of the duogrid).
__device__ __forceinline__ long band_source(const RouteTable& rt, int f, int ti, int tj, int n) {
  const int m = n + 6;
  int d, c, k;
  if (tj < kHalo) { d = kW; c = tj; k = ti - kHalo; }
  else if (tj >= m - kHalo) { d = kE; c = tj - (m - kHalo); k = ti - kHalo; }
  else if (ti < kHalo) { d = kS; c = ti; k = tj - kHalo; }
  else { d = kN; c = ti - (m - kHalo); k = tj - kHalo; }
  const int r = rt.r[f * 4 + d];
  const int kk = route_rev(r) ? n - 1 - k : k;
  int si, sj;
  switch (route_side(r)) {
    case kE: si = kHalo + kk; sj = m - 6 + c; break;
    case kW: si = kHalo + kk; sj = kHalo + c; break;
    case kN: si = m - 6 + c; sj = kHalo + kk; break;
    default: si = kHalo + c; sj = kHalo + kk; break;
  }
  return cell(route_nb(r), si, sj, m);
}

// One thread per halo cell: two source cells and two weights (the linear
// kinked -> extended remap along the band; corners take the band cell of row
// 3 / M-4).  Location indices are clamped into the band so that no read can go
// out of bounds (k_check_tables has rejected tables that would need it).
template <typename T>
__global__ void k_build_halo(int n, const T* coef, const int* li, const int* lj, RouteTable rt, int2* src,
                             T* w) {
  const int m = n + 6, nh = halo_count(m);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 6 * nh) return;
  const int f = k / nh, id = k - f * nh;
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
  int bi = i;
  const int bj = j;
  if ((i < kHalo || i >= m - kHalo) && (j < kHalo || j >= m - kHalo)) bi = i < kHalo ? kHalo : m - kHalo - 1;
  const long ob = cell(f, bi, bj, m);
  const bool along_i = (bj < kHalo || bj >= m - kHalo);
  int loc = along_i ? li[ob] : lj[ob];
  loc = min(max(loc, kHalo), m - kHalo - 2);
  long s0, s1;
  if (along_i) {
    s0 = band_source(rt, f, loc, bj, n);
    s1 = band_source(rt, f, loc + 1, bj, n);
  } else {
    s0 = band_source(rt, f, bi, loc, n);
    s1 = band_source(rt, f, bi, loc + 1, n);
  }
  src[k] = make_int2((int)s0, (int)s1);
  w[2 * k] = coef[2 * ob];
  w[2 * k + 1] = coef[2 * ob + 1];
}

// The checks of bt_plan_create on the device, one thread per cell of the
// (6, M, M) arrays: inner / outer must be the exact interior / halo masks
// (kBadMask), and at a halo cell the k2e location the remap reads (loc_i
// along the W/E bands, loc_j along the S/N bands, the band cell of row 3 /
// M-4 at corners) must lie in [3, M-5] (kBadLocation).
template <typename T>
__global__ void k_check_tables(int n, const int* li, const int* lj, const T* inner, const T* outer,
                               unsigned* status) {
  const int m = n + 6;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 6 * m * m) return;
  const int f = k / (m * m), r = k - f * m * m, i = r / m, j = r - (r / m) * m;
  const bool in = is_interior(i, j, m);
  const T want = in ? T(1) : T(0);
  if (inner[k] != want || outer[k] != T(1) - want) atomicOr(status, (unsigned)kBadMask);
  if (in) return;
  int bi = i;
  if ((i < kHalo || i >= m - kHalo) && (j < kHalo || j >= m - kHalo)) bi = i < kHalo ? kHalo : m - kHalo - 1;
  const long ob = cell(f, bi, j, m);
  const int loc = (j < kHalo || j >= m - kHalo) ? li[ob] : lj[ob];
  if (loc < kHalo || loc > m - kHalo - 2) atomicOr(status, (unsigned)kBadLocation);
}

// Check the constant set once per device (see the file comment); waits for the result.
template <typename T>
int check_tables_once(unsigned char* base, const bt_grid_desc& d, cudaStream_t s) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return set_error(BT_ECUDA, "bt_round_noalloc: cudaGetDevice failed");
  const void* cs[17] = {d.dzph_x, d.dzph_y, d.rdx, d.rdy, d.a_f, d.k2e_coef, d.loc_i_local, d.loc_j_local,
                        d.a_c2l, d.a_l2c, d.inner, d.outer, d.a_gct, d.a_sina, d.rda, d.c_dy, d.d_dx};
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const CheckedDesc& c = g_checked[dev];
    if (c.valid && c.n == d.n && c.dtype == d.dtype && std::memcmp(c.c, cs, sizeof(cs)) == 0) return BT_OK;
  }
  unsigned* status = (unsigned*)base;
  const int m = d.n + 6, total = 6 * m * m, th = 256;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(unsigned), s);
  if (e == cudaSuccess) {
    k_check_tables<T><<<(total + th - 1) / th, th, 0, s>>>(d.n, d.loc_i_local, d.loc_j_local, (const T*)d.inner,
                                                           (const T*)d.outer, status);
    e = cudaGetLastError();
  }
  unsigned st = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&st, status, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_error(BT_ECUDA, std::string("bt_round_noalloc: table check: ") + cudaGetErrorString(e));
  if (st & kBadMask)
    return set_error(BT_ENOTSUP, "bt_round_noalloc: inner/outer must be the interior/halo masks of duogrid.py:159-190");
  if (st & kBadLocation) return set_error(BT_EINVAL, "bt_round_noalloc: k2e location table out of range at a halo cell");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  CheckedDesc& c = g_checked[dev];
  c.valid = true;
  c.n = d.n;
  c.dtype = d.dtype;
  std::memcpy(c.c, cs, sizeof(cs));
  return BT_OK;
}

template <typename T>
StageIO<T> io_of(const T* h, const T* u, const T* v, const T* hp, const T* up, const T* vp, T* ho, T* uo, T* vo,
                 T* fx, double dt, double beta, int stored, int last) {
  StageIO<T> io;
  io.h = h;
  io.u = u;
  io.v = v;
  io.hp = hp;
  io.up = up;
  io.vp = vp;
  io.h_out = ho;
  io.u_out = uo;
  io.v_out = vo;
  io.fx = fx;
  io.dt = (T)dt;
  io.beta = (T)beta;
  io.stored_halo = stored;
  io.last = last;
  return io;
}

template <typename T>
int run_noalloc(unsigned char* base, const bt_grid_desc& d, const bt_state_in& in, const bt_state_out& out, int nbb,
                double dtb, int rk, cudaStream_t s) {
  const int n = d.n, m = n + 6, nh = halo_count(m);
  // face cache blocks of the 8 x 16 tiles this entry point runs
  const size_t fe = (size_t)6 * m * m,
               face = (size_t)6 * ((n + 7) / 8) * ((n + 15) / 16) * TileShape<8, 16>::fW;
  const size_t o_src = kStatusBytes;
  const size_t o_w = o_src + align256((size_t)6 * nh * sizeof(int2));
  const size_t o_f = o_w + align256((size_t)6 * nh * 2 * sizeof(T));
  const int nfields = rk == 2 ? 3 : 6;
  const size_t o_fx = o_f + align256((size_t)nfields * fe * sizeof(T));
  const size_t need = o_fx + align256(face * sizeof(T));
  if (need > kScratchBytes)
    return set_error(BT_EINVAL, "bt_round_noalloc: N = " + std::to_string(n) + " needs " + std::to_string(need) +
                                    " bytes of scratch, more than the library's fixed " +
                                    std::to_string(kScratchBytes) + "; use bt_plan_create/bt_round");
  const int rc = check_tables_once<T>(base, d, s);
  if (rc != BT_OK) return rc;
  int2* hsrc = (int2*)(base + o_src);
  T* hw = (T*)(base + o_w);
  T* F = (T*)(base + o_f);
  T* fx = (T*)(base + o_fx);
  const RouteTable rt = make_routes();
  const int cells = 6 * nh, th = 256;
  k_build_halo<T><<<(cells + th - 1) / th, th, 0, s>>>(n, (const T*)d.k2e_coef, d.loc_i_local, d.loc_j_local, rt,
                                                       hsrc, hw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(BT_ECUDA, std::string("bt_round_noalloc: ") + cudaGetErrorString(e));

  Geo<T> g;
  g.n = n;
  g.m = m;
  g.nh = nh;
  g.dzph_x = (const T*)d.dzph_x;
  g.dzph_y = (const T*)d.dzph_y;
  g.rdx = (const T*)d.rdx;
  g.rdy = (const T*)d.rdy;
  g.a_f = (const T*)d.a_f;
  g.c2l = (const T*)d.a_c2l;
  g.l2c = (const T*)d.a_l2c;
  g.gct = (const T*)d.a_gct;
  g.sina = (const T*)d.a_sina;
  g.rda = (const T*)d.rda;
  g.c_dy = (const T*)d.c_dy;
  g.d_dx = (const T*)d.d_dx;
  g.hsrc = hsrc;
  g.hw = hw;
  g.cblk = nullptr;  // no prepared constant blocks: phase UV reads the constant arrays
  g.cblk_ti = g.cblk_tj = 0;
  for (int k = 0; k < 24; ++k) g.route[k] = rt.r[k];

  T* Y[3] = {F, F + fe, F + 2 * fe};
  T* Z[3] = {F + 3 * fe, F + 4 * fe, F + 5 * fe};
  T* X[3] = {(T*)out.h0, (T*)out.ub, (T*)out.vb};
  const T* X0[3] = {(const T*)in.h0, (const T*)in.ub, (const T*)in.vb};
  const T* B0[3] = {(const T*)in.h0p, (const T*)in.ubp, (const T*)in.vbp};
  const TileCfg tile{8, 16};
  auto stage = [&](const StageIO<T>& io) {
    cudaError_t r = launch_phase_h<T>(g, io, tile, s);
    return r == cudaSuccess ? launch_phase_uv<T>(g, io, tile, s) : r;
  };
  for (int step = 0; step < nbb && e == cudaSuccess; ++step) {
    const T* const* cur = step == 0 ? X0 : (const T* const*)X;
    const T* const* bs = step == 0 ? B0 : (const T* const*)X;
    const int stored = step == 0 ? 1 : 0;
    if (rk == 2) {
      e = stage(io_of<T>(cur[0], cur[1], cur[2], bs[0], bs[1], bs[2], Y[0], Y[1], Y[2], fx, dtb / 2.0, 0.0,
                         stored, 0));
      if (e == cudaSuccess)
        e = stage(io_of<T>(Y[0], Y[1], Y[2], bs[0], bs[1], bs[2], X[0], X[1], X[2], fx, dtb, 0.0, 0, 1));
    } else {
      e = stage(io_of<T>(cur[0], cur[1], cur[2], bs[0], bs[1], bs[2], Y[0], Y[1], Y[2], fx, dtb / 3.0, 1.0,
                         stored, 0));
      if (e == cudaSuccess)
        e = stage(io_of<T>(Y[0], Y[1], Y[2], bs[0], bs[1], bs[2], Z[0], Z[1], Z[2], fx, dtb / 2.0, 1.0, 0, 0));
      if (e == cudaSuccess)
        e = stage(io_of<T>(Z[0], Z[1], Z[2], bs[0], bs[1], bs[2], X[0], X[1], X[2], fx, dtb, 1.0, 0, 1));
    }
  }
  if (e == cudaSuccess && out.diag[0]) {
    T* const* L = rk == 2 ? Y : Z;
    e = launch_fill_halo<T>(g, L[0], L[1], L[2], s);
    if (e == cudaSuccess) {
      DiagOut<T> dg;
      T** dp = (T**)&dg;
      for (int k = 0; k < 10; ++k) dp[k] = (T*)out.diag[k];
      e = launch_diag<T>(g, L[0], L[1], L[2], dg, s);
    }
  }
  if (e == cudaSuccess) e = launch_fill_halo<T>(g, X[0], X[1], X[2], s);
  if (e != cudaSuccess) return set_error(BT_ECUDA, std::string("bt_round_noalloc: ") + cudaGetErrorString(e));
  return BT_OK;
}

// Per-device set-up, once: the array's device address and the kernels' shared-memory opt-in.
int setup_device(int dtype, unsigned char** base) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(BT_ECUDA, std::string("bt_round_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return set_error(BT_ENOTSUP, "bt_round_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
      return set_error(BT_ECUDA, std::string("bt_round_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  bool& primed = dtype == BT_F64 ? g_primed_f64[dev] : g_primed_f32[dev];
  if (!primed) {
    e = dtype == BT_F64 ? prime_kernels<double>() : prime_kernels<float>();
    if (e != cudaSuccess)
      return set_error(BT_ECUDA, std::string("bt_round_noalloc: kernel attributes: ") + cudaGetErrorString(e));
    primed = true;
  }
  *base = (unsigned char*)g_scratch_addr[dev];
  return BT_OK;
}

}  // namespace
}  // namespace bt

using namespace bt;

extern "C" int bt_round_noalloc(const bt_grid_desc* desc, const bt_state_in* in, const bt_state_out* out, int nbb,
                                double dtb, int rk, void* stream) {
  if (!desc || !in || !out) return set_error(BT_EINVAL, "bt_round_noalloc: NULL argument");
  if (desc->n < 4) return set_error(BT_EINVAL, "bt_round_noalloc: n must be >= 4");
  if (desc->dtype != BT_F64 && desc->dtype != BT_F32)
    return set_error(BT_EINVAL, "bt_round_noalloc: dtype must be BT_F64 or BT_F32");
  if (rk != 2 && rk != 3) return set_error(BT_EINVAL, "bt_round_noalloc: rk must be 2 or 3");
  if (nbb < 1) return set_error(BT_EINVAL, "bt_round_noalloc: nbb must be >= 1");
  const void* cs[17] = {desc->dzph_x, desc->dzph_y, desc->rdx, desc->rdy, desc->a_f, desc->k2e_coef,
                        desc->loc_i_local, desc->loc_j_local, desc->a_c2l, desc->a_l2c, desc->inner, desc->outer,
                        desc->a_gct, desc->a_sina, desc->rda, desc->c_dy, desc->d_dx};
  for (const void* c : cs)
    if (!c) return set_error(BT_EINVAL, "bt_round_noalloc: NULL constant pointer");
  if (!matrices_aligned(desc))
    return set_error(BT_EINVAL, "bt_round_noalloc: a_c2l, a_l2c and a_gct must be 16-byte aligned");
  const void* ins[6] = {in->h0, in->h0p, in->ub, in->vb, in->ubp, in->vbp};
  for (const void* q : ins) {
    if (!q) return set_error(BT_EINVAL, "bt_round_noalloc: NULL input field");
    if (q == out->h0 || q == out->ub || q == out->vb)
      return set_error(BT_EINVAL, "bt_round_noalloc: output fields must not alias the inputs");
  }
  if (!out->h0 || !out->ub || !out->vb) return set_error(BT_EINVAL, "bt_round_noalloc: NULL output field");
  if (out->diag[0])
    for (int k = 1; k < 10; ++k)
      if (!out->diag[k]) return set_error(BT_EINVAL, "bt_round_noalloc: diag outputs must be all set or diag[0] NULL");
  unsigned char* base = nullptr;
  const int rc = setup_device(desc->dtype, &base);
  if (rc != BT_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  return desc->dtype == BT_F64 ? run_noalloc<double>(base, *desc, *in, *out, nbb, dtb, rk, s)
                               : run_noalloc<float>(base, *desc, *in, *out, nbb, dtb, rk, s);
}
