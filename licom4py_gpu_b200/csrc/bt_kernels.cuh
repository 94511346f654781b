// bt_kernels.cuh - sm_100a kernels of the barotropic duogrid solver and their launchers.
//
// Included by bt_kernels_f64.cu (float64 drop-in, compiled with -fmad=false so
// the arithmetic rounds like the reference term by term) and bt_kernels_f32.cu
// (float32 precision form, FMA contraction allowed), each instantiating one type.
//
// Per RK stage two tile kernels run back to back (phase H, phase UV); each CTA
// stages one tile of one face plus its 3-cell stencil halo in shared memory
// (cross-shaped region, corners skipped), computes the C/D-grid face
// quantities once per face and the cell updates from them.  The whole
// member (6 faces) is one launch; halos across face edges are gathered
// inside the tile loader (bt_stencil.cuh), so no separate exchange kernel
// runs between phases.

#pragma once

#include <algorithm>
#include <atomic>

#include "bt_launch.cuh"

namespace bt {

constexpr int kThreads = kTileThreads;


// FP: the full-interior-tile path compiled in (multi-wave launches), else
// every tile runs the edge path (one-wave launches: half the code to fetch).
template <typename T, int TI, int TJ, bool FP>
__global__ void __launch_bounds__(kThreads, PhaseBlocks<T, FP>::value) k_phase_h(Geo<T> g, StageIO<T> io, Tiling t) {
  extern __shared__ __align__(16) unsigned char smraw[];
  release_dependents();
  const TileBox b = tile_box(t, g.n, blockIdx.x);
  tile_h<T, TI, TJ, FP>(g, io, b, reinterpret_cast<T*>(smraw));
}

template <typename T, int TI, int TJ, bool FP>
__global__ void __launch_bounds__(kThreads, PhaseBlocksUV<T>::value) k_phase_uv(Geo<T> g, StageIO<T> io, Tiling t) {
  extern __shared__ __align__(16) unsigned char smraw[];
  release_dependents();
  const TileBox b = tile_box(t, g.n, blockIdx.x);
  tile_uv<T, TI, TJ, FP>(g, io, b, reinterpret_cast<T*>(smraw));
}

// One whole round of one member in a single cooperative launch: every CTA
// walks its tiles of a phase, then all CTAs meet at a grid barrier.  Before
// waiting at the barrier a CTA already issues the next phase's prologue for
// its first tile (constants by cp.async, halo descriptors), so those loads
// overlap the barrier.  The loop runs per RK stage (phase H, barrier, phase
// UV, barrier) so the two phases' gather states are never live together.
template <typename T, int TI, int TJ>
__global__ void __launch_bounds__(kThreads, 3) k_round(RoundArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ StageIO<T> s_io[2];  // stage pointers, alternating between consecutive stages
  T* sm = reinterpret_cast<T*>(smraw);
  const int ntiles = 6 * a.t.tiles_per_face();
  const int nst = a.rk == 2 ? 2 : 3;
  const int nstage = a.nbb * nst;
  const int t0 = blockIdx.x;
  unsigned gen = 0;
  EdgeCnt cnt;
  int P = 0;
  if (threadIdx.x == 0) s_io[0] = round_stage(a, a.step0, 0);
  __syncthreads();
  // phase H of stage 0: the first tile's prologue
  Gather<T, TI, TJ, false> gh;
  if (t0 < ntiles) tile_h_pro<T, TI, TJ>(a.g, s_io[0], tile_box(a.t, a.g.n, t0), sm, gh, cnt, P);
  for (int sg = 0; sg < nstage; ++sg) {
    const StageIO<T>& io = s_io[sg & 1];
    int k = 0;
    for (int tile = t0; tile < ntiles; tile += gridDim.x, ++k) {
      const TileBox b = tile_box(a.t, a.g.n, tile);
      if (k > 0) tile_h_pro<T, TI, TJ>(a.g, io, b, sm, gh, cnt, P);
      tile_h_main<T, TI, TJ>(a.g, io, b, sm, gh, cnt, P);
      __syncthreads();
    }
    Gather<T, TI, TJ, true> gu;
    if (t0 < ntiles) tile_uv_pro<T, TI, TJ>(a.g, io, tile_box(a.t, a.g.n, t0), sm, gu, cnt, P);
    if (!grid_barrier(a.bar, gen, a.err, a.spin_limit)) {
      cp_async_wait_all();  // no copy may be left in flight when the CTA leaves
      return;
    }
    k = 0;
    for (int tile = t0; tile < ntiles; tile += gridDim.x, ++k) {
      const TileBox b = tile_box(a.t, a.g.n, tile);
      if (k > 0) tile_uv_pro<T, TI, TJ>(a.g, io, b, sm, gu, cnt, P);
      tile_uv_main<T, TI, TJ>(a.g, io, b, sm, gu, cnt, P);
      __syncthreads();
    }
    if (sg + 1 < nstage) {
      if (threadIdx.x == 0) s_io[(sg + 1) & 1] = round_stage(a, a.step0 + (sg + 1) / nst, (sg + 1) % nst);
      __syncthreads();
      if (t0 < ntiles) tile_h_pro<T, TI, TJ>(a.g, s_io[(sg + 1) & 1], tile_box(a.t, a.g.n, t0), sm, gh, cnt, P);
    }
    if (!grid_barrier(a.bar, gen, a.err, a.spin_limit)) {
      cp_async_wait_all();
      return;
    }
  }
}

// Tile constant blocks: word w < uConstWords of tile t's block is what
// tile_uv_consts stages at shared-memory word uG + w for that tile (gct, sina,
// rda, rdx, rdy, a_f of its cells, c_dy of its x faces, d_dx of its y faces);
// then dzph_x of its x faces and dzph_y of its y faces, indexed like phase H's
// shared-memory planes.  Positions outside a partial tile and the padding are zero.
template <typename T, int TI, int TJ>
__global__ void __launch_bounds__(kThreads) k_const_blocks(Geo<T> g, Tiling t, T* out) {
  using S = TileShape<TI, TJ>;
  const long total = 6L * t.nti * t.ntj * S::cW;
  const int m = g.m;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total; k += (long)gridDim.x * blockDim.x) {
    const int tile = (int)(k / S::cW), w = (int)(k - (long)tile * S::cW), o = S::uG + w;
    const TileBox b = tile_box_at(t, g.n, tile);
    T v = T(0);
    if (w >= S::bDZX) {
      if (w < S::bDZY) {
        const int e = w - S::bDZX, a = e / TJ, q = e % TJ;
        if (a <= b.ni && q < b.nj) v = g.dzph_x[cell(b.f, b.i0 + a, b.j0 + q, m)];
      } else if (w < S::bDZY + S::FY) {
        const int e = w - S::bDZY, r = e / (TJ + 1), qq = e % (TJ + 1);
        if (r < b.ni && qq <= b.nj) v = g.dzph_y[cell(b.f, b.i0 + r, b.j0 + qq, m)];
      }
    } else if (o < S::uSN) {
      const int e = (o - S::uG) / 4, comp = (o - S::uG) % 4, a = e / TJ, q = e % TJ;
      if (a < b.ni && q < b.nj) v = g.gct[4 * cell(b.f, b.i0 + a, b.j0 + q, m) + comp];
    } else if (o < S::uAF + S::C) {
      const int arr = (o - S::uSN) / S::C, e = (o - S::uSN) % S::C, a = e / TJ, q = e % TJ;
      if (a < b.ni && q < b.nj) {
        const long c = cell(b.f, b.i0 + a, b.j0 + q, m);
        v = arr == 0 ? g.sina[c] : arr == 1 ? g.rda[c] : arr == 2 ? g.rdx[c] : arr == 3 ? g.rdy[c] : g.a_f[c];
      }
    } else if (o >= S::uCDY && o < S::uCDY + S::FX) {
      const int e = o - S::uCDY, a = e / TJ, q = e % TJ;
      if (a <= b.ni && q < b.nj) v = g.c_dy[cell(b.f, b.i0 + a, b.j0 + q, m)];
    } else if (o >= S::uDDX && o < S::uDDX + S::FY) {
      const int e = o - S::uDDX, r = e / (TJ + 1), qq = e % (TJ + 1);
      if (r < b.ni && qq <= b.nj) v = g.d_dx[cell(b.f, b.i0 + r, b.j0 + qq, m)];
    }
    out[k] = v;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_fill_halo(Geo<T> g, T* h, T* u, T* v) {
  wait_prior_grid();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < 6 * g.nh) fill_halo_cell(g, h, u, v, k);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_diag(Geo<T> g, const T* h, const T* u, const T* v,
                                                   DiagOut<T> d) {
  wait_prior_grid();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = g.m;
  if (k >= 6 * m * m) return;
  const int f = k / (m * m);
  const int r = k - f * m * m;
  diag_cell(g, h, u, v, d, f, r / m, r % m);
}

#ifdef BT_DEFINE_COMMON
bool tile_cfg_supported(TileCfg c) {
  return (c.tj == 32 && (c.ti == 7 || c.ti == 8 || c.ti == 15 || c.ti == 16)) ||
         (c.tj == 16 && (c.ti == 8 || c.ti == 16));
}

namespace {
template <int TI, int TJ>
size_t face_cache_elems_tile(int n) {
  const size_t nti = (n + TI - 1) / TI, ntj = (n + TJ - 1) / TJ;
  return 6 * nti * ntj * (size_t)TileShape<TI, TJ>::fW;
}
}  // namespace

namespace {
template <int TI, int TJ>
size_t const_block_elems_tile(int n) {
  const size_t nti = (n + TI - 1) / TI, ntj = (n + TJ - 1) / TJ;
  return 6 * nti * ntj * (size_t)TileShape<TI, TJ>::cW;
}
}  // namespace

size_t const_block_elems(TileCfg c, int n) {
  if (c.ti == 7 && c.tj == 32) return const_block_elems_tile<7, 32>(n);
  if (c.ti == 8 && c.tj == 32) return const_block_elems_tile<8, 32>(n);
  if (c.ti == 15 && c.tj == 32) return const_block_elems_tile<15, 32>(n);
  if (c.ti == 16 && c.tj == 32) return const_block_elems_tile<16, 32>(n);
  if (c.ti == 8 && c.tj == 16) return const_block_elems_tile<8, 16>(n);
  if (c.ti == 16 && c.tj == 16) return const_block_elems_tile<16, 16>(n);
  return 0;
}

size_t face_cache_elems(int n) {
  const size_t s[6] = {face_cache_elems_tile<7, 32>(n), face_cache_elems_tile<8, 32>(n),
                       face_cache_elems_tile<15, 32>(n), face_cache_elems_tile<16, 32>(n),
                       face_cache_elems_tile<8, 16>(n), face_cache_elems_tile<16, 16>(n)};
  return *std::max_element(s, s + 6);
}

Tiling make_tiling(TileCfg c, int n) {
  Tiling t;
  t.ti = c.ti;
  t.tj = c.tj;
  t.nti = (n + c.ti - 1) / c.ti;
  t.ntj = (n + c.tj - 1) / c.tj;
  return t;
}
#endif

namespace {

template <typename T, int TI, int TJ, bool UV>
size_t tile_smem() {
  using S = TileShape<TI, TJ>;
  return sizeof(T) * (UV ? S::kWordsUV : S::kWordsH) + sizeof(int) * kItemWords;
}

// The persistent kernel runs both phases in one allocation: the larger of the two.
template <typename T, int TI, int TJ>
size_t round_smem() {
  return std::max(tile_smem<T, TI, TJ, false>(), tile_smem<T, TI, TJ, true>());
}

// CTAs of one phase kernel (edge-only build) that fit on each device at once,
// recorded by prime_tile at plan creation (0 = not recorded yet).
constexpr int kMaxDevices = 64;
template <typename T, int TI, int TJ, bool UV>
std::atomic<int>* wave_slots() {  // relaxed: plans on several host threads may record them at once
  static std::atomic<int> slots[kMaxDevices];
  return slots;
}

template <typename T, int TI, int TJ, bool UV>
cudaError_t record_wave_slots() {
  int dev, sms, per_sm;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaSuccess;  // the launch then keeps the full-tile path
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  auto kern = UV ? k_phase_uv<T, TI, TJ, false> : k_phase_h<T, TI, TJ, false>;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, tile_smem<T, TI, TJ, UV>())) !=
      cudaSuccess)
    return e;
  wave_slots<T, TI, TJ, UV>()[dev].store(sms * per_sm, std::memory_order_relaxed);
  return cudaSuccess;
}

// Opt in to more than 48 KB of dynamic shared memory and record the wave slots
// (done at plan creation, never during stream capture).
template <typename T, int TI, int TJ>
cudaError_t prime_tile() {
  cudaError_t e;
  for (auto k : {k_phase_h<T, TI, TJ, true>, k_phase_h<T, TI, TJ, false>})
    if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tile_smem<T, TI, TJ, false>())) != cudaSuccess)
      return e;
  for (auto k : {k_phase_uv<T, TI, TJ, true>, k_phase_uv<T, TI, TJ, false>})
    if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tile_smem<T, TI, TJ, true>())) != cudaSuccess)
      return e;
  e = cudaFuncSetAttribute(k_round<T, TI, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)round_smem<T, TI, TJ>());
  if (e != cudaSuccess) return e;
  if ((e = record_wave_slots<T, TI, TJ, false>()) != cudaSuccess) return e;
  return record_wave_slots<T, TI, TJ, true>();
}

// Co-resident grid for the persistent kernel (at most one CTA per tile).
template <typename T, int TI, int TJ>
cudaError_t launch_round_tile(RoundArgs<T> a, int max_ctas, cudaStream_t s, int* grid_out) {
  const size_t smem = round_smem<T, TI, TJ>();
  int dev, sms, per_sm;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_round<T, TI, TJ>, kThreads, smem)) !=
      cudaSuccess)
    return e;
  a.t = make_tiling({TI, TJ}, a.g.n);
  int grid = std::min(per_sm * sms, 6 * a.t.tiles_per_face());
  if (max_ctas > 0) grid = std::min(grid, max_ctas);
  if (grid < 1) return cudaErrorInvalidConfiguration;
  if (grid_out) *grid_out = grid;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)k_round<T, TI, TJ>, dim3(grid), dim3(kThreads), args, smem, s);
}

// Whether a phase launch at n cells per face edge runs the full-tile kernel:
// forced by full_tiles >= 0, else by size (the edge-only kernel when the
// launch's CTAs all fit on the current device at once).
template <typename T, int TI, int TJ, bool UV>
bool full_path(int n, int full_tiles) {
  if (full_tiles >= 0) return full_tiles != 0;
  int dev = -1;
  int slots = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxDevices)
    slots = wave_slots<T, TI, TJ, UV>()[dev].load(std::memory_order_relaxed);
  return !(slots > 0 && 6 * make_tiling({TI, TJ}, n).tiles_per_face() <= slots);
}

template <typename T, int TI, int TJ, bool UV>
cudaError_t launch_tile(const Geo<T>& g, const StageIO<T>& io, cudaStream_t s, int full_tiles) {
  const size_t smem = tile_smem<T, TI, TJ, UV>();
  const Tiling t = make_tiling({TI, TJ}, g.n);
  const bool fp = full_path<T, TI, TJ, UV>(g.n, full_tiles);
  auto kern = UV ? (fp ? k_phase_uv<T, TI, TJ, true> : k_phase_uv<T, TI, TJ, false>)
                 : (fp ? k_phase_h<T, TI, TJ, true> : k_phase_h<T, TI, TJ, false>);
  // programmatic dependent launch: the kernel's constant prologue overlaps the
  // previous kernel's tail; it waits (griddepcontrol.wait) before reading state
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(6 * t.tiles_per_face());
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, g, io, t);
}

template <typename T, bool UV>
cudaError_t dispatch(const Geo<T>& g, const StageIO<T>& io, TileCfg c, cudaStream_t s, int full_tiles) {
  if (c.ti == 7 && c.tj == 32) return launch_tile<T, 7, 32, UV>(g, io, s, full_tiles);
  if (c.ti == 8 && c.tj == 32) return launch_tile<T, 8, 32, UV>(g, io, s, full_tiles);
  if (c.ti == 15 && c.tj == 32) return launch_tile<T, 15, 32, UV>(g, io, s, full_tiles);
  if (c.ti == 16 && c.tj == 32) return launch_tile<T, 16, 32, UV>(g, io, s, full_tiles);
  if (c.ti == 8 && c.tj == 16) return launch_tile<T, 8, 16, UV>(g, io, s, full_tiles);
  if (c.ti == 16 && c.tj == 16) return launch_tile<T, 16, 16, UV>(g, io, s, full_tiles);
  return cudaErrorInvalidValue;
}

}  // namespace

template <typename T>
cudaError_t launch_round(const RoundArgs<T>& a, TileCfg c, int max_ctas, cudaStream_t s, int* grid_out) {
  if (c.ti == 7 && c.tj == 32) return launch_round_tile<T, 7, 32>(a, max_ctas, s, grid_out);
  if (c.ti == 8 && c.tj == 32) return launch_round_tile<T, 8, 32>(a, max_ctas, s, grid_out);
  if (c.ti == 15 && c.tj == 32) return launch_round_tile<T, 15, 32>(a, max_ctas, s, grid_out);
  if (c.ti == 16 && c.tj == 32) return launch_round_tile<T, 16, 32>(a, max_ctas, s, grid_out);
  if (c.ti == 8 && c.tj == 16) return launch_round_tile<T, 8, 16>(a, max_ctas, s, grid_out);
  if (c.ti == 16 && c.tj == 16) return launch_round_tile<T, 16, 16>(a, max_ctas, s, grid_out);
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t prime_kernels() {
  cudaError_t e;
  if ((e = prime_tile<T, 7, 32>()) != cudaSuccess) return e;
  if ((e = prime_tile<T, 8, 32>()) != cudaSuccess) return e;
  if ((e = prime_tile<T, 15, 32>()) != cudaSuccess) return e;
  if ((e = prime_tile<T, 16, 32>()) != cudaSuccess) return e;
  if ((e = prime_tile<T, 8, 16>()) != cudaSuccess) return e;
  return prime_tile<T, 16, 16>();
}

template <typename T>
int phase_full_paths(TileCfg c, int n, int full_tiles) {
#define BT_FP_BITS(TI, TJ) \
  if (c.ti == TI && c.tj == TJ) \
    return (full_path<T, TI, TJ, false>(n, full_tiles) ? 1 : 0) | (full_path<T, TI, TJ, true>(n, full_tiles) ? 2 : 0);
  BT_FP_BITS(7, 32)
  BT_FP_BITS(8, 32)
  BT_FP_BITS(15, 32)
  BT_FP_BITS(16, 32)
  BT_FP_BITS(8, 16)
  BT_FP_BITS(16, 16)
#undef BT_FP_BITS
  return -1;
}

template <typename T>
cudaError_t launch_phase_h(const Geo<T>& g, const StageIO<T>& io, TileCfg cfg, cudaStream_t s, int full_tiles) {
  return dispatch<T, false>(g, io, cfg, s, full_tiles);
}

template <typename T>
cudaError_t launch_phase_uv(const Geo<T>& g, const StageIO<T>& io, TileCfg cfg, cudaStream_t s, int full_tiles) {
  return dispatch<T, true>(g, io, cfg, s, full_tiles);
}

template <typename T, int TI, int TJ>
cudaError_t launch_const_blocks_tile(const Geo<T>& g, T* out, cudaStream_t s) {
  const Tiling t = make_tiling({TI, TJ}, g.n);
  const long total = 6L * t.nti * t.ntj * TileShape<TI, TJ>::cW;
  const int grid = (int)std::min<long>((total + kThreads - 1) / kThreads, 148L * 16);
  k_const_blocks<T, TI, TJ><<<grid, kThreads, 0, s>>>(g, t, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_const_blocks(const Geo<T>& g, TileCfg c, T* out, cudaStream_t s) {
  if (c.ti == 7 && c.tj == 32) return launch_const_blocks_tile<T, 7, 32>(g, out, s);
  if (c.ti == 8 && c.tj == 32) return launch_const_blocks_tile<T, 8, 32>(g, out, s);
  if (c.ti == 15 && c.tj == 32) return launch_const_blocks_tile<T, 15, 32>(g, out, s);
  if (c.ti == 16 && c.tj == 32) return launch_const_blocks_tile<T, 16, 32>(g, out, s);
  if (c.ti == 8 && c.tj == 16) return launch_const_blocks_tile<T, 8, 16>(g, out, s);
  if (c.ti == 16 && c.tj == 16) return launch_const_blocks_tile<T, 16, 16>(g, out, s);
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_fill_halo(const Geo<T>& g, T* h, T* u, T* v, cudaStream_t s) {
  const int total = 6 * g.nh;
  k_fill_halo<T><<<(total + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, h, u, v);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_diag(const Geo<T>& g, const T* h, const T* u, const T* v, const DiagOut<T>& d,
                        cudaStream_t s) {
  const int total = 6 * g.m * g.m;
  k_diag<T><<<(total + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, h, u, v, d);
  return cudaGetLastError();
}

#define BT_INSTANTIATE(T)                                                                           \
  template cudaError_t prime_kernels<T>();                                                          \
  template int phase_full_paths<T>(TileCfg, int, int);                                              \
  template cudaError_t launch_phase_h<T>(const Geo<T>&, const StageIO<T>&, TileCfg, cudaStream_t, int);  \
  template cudaError_t launch_phase_uv<T>(const Geo<T>&, const StageIO<T>&, TileCfg, cudaStream_t, int); \
  template cudaError_t launch_fill_halo<T>(const Geo<T>&, T*, T*, T*, cudaStream_t);                \
  template cudaError_t launch_const_blocks<T>(const Geo<T>&, TileCfg, T*, cudaStream_t);               \
  template cudaError_t launch_round<T>(const RoundArgs<T>&, TileCfg, int, cudaStream_t, int*);      \
  template cudaError_t launch_diag<T>(const Geo<T>&, const T*, const T*, const T*, const DiagOut<T>&, \
                                      cudaStream_t);

}  // namespace bt
