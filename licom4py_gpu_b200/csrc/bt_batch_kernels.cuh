// bt_batch_kernels.cuh - kernels and launchers of the batched rounds
// (types in bt_batch.cuh).  Included by bt_batch_f64.cu / bt_batch_f32.cu,
// each compiled with the FMA setting of its type like the single-member kernels.

#pragma once

#include <algorithm>
#include <atomic>

#include "bt_batch.cuh"

namespace bt {

__device__ __forceinline__ Tiling make_tiling_dev(int ti, int tj, int n) {
  Tiling t;
  t.ti = ti;
  t.tj = tj;
  t.nti = (n + ti - 1) / ti;
  t.ntj = (n + tj - 1) / tj;
  return t;
}

// Largest k with off[k] <= item (off non-decreasing, off[0] = 0 <= item < off[count]).
__device__ __forceinline__ int member_of(const int* off, int count, int item) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= item)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The same search by one warp: each round the 32 lanes test 32 evenly spaced
// offsets of the remaining range at once, so a list of up to 32 members takes
// one load round trip and up to 1024 two.  Every lane returns the result.
__device__ __forceinline__ int member_of_warp(const int* off, int count, int item) {
  const int lane = threadIdx.x & 31;
  int lo = 0, hi = count;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const int step = (hi - lo + 31) >> 5;
    const int idx = lo + lane * step;
    const bool le = idx < hi && __ldg(off + idx) <= item;
    const unsigned m = __ballot_sync(0xffffffffu, le);  // lane 0 always set: off[lo] <= item
    const int last = 31 - __clz(m);
    lo += last * step;
    hi = min(hi, lo + step);
  }
  return lo;
}

// Stage pointers of member k at (substep, stage); the schedule of
// barotr.py:41-87 as in the single-member round.
template <typename T>
__device__ StageIO<T> member_stage(const MemberDesc<T>& d, int rk, int step, int st) {
  StageIO<T> io;
  const T* const* cur = step == 0 ? d.x0 : (const T* const*)d.x;
  const T* const* base = step == 0 ? d.b0 : (const T* const*)d.x;
  const int nst = rk == 2 ? 2 : 3;
  const T* const* in = st == 0 ? cur : (st == 1 ? (const T* const*)d.y : (const T* const*)d.z);
  T* const* out = st == nst - 1 ? d.x : (st == 0 ? d.y : d.z);
  io.h = in[0];
  io.u = in[1];
  io.v = in[2];
  io.hp = base[0];
  io.up = base[1];
  io.vp = base[2];
  io.h_out = out[0];
  io.u_out = out[1];
  io.v_out = out[2];
  io.fx = d.fx;
  double dt;
  if (rk == 2) {
    dt = st == 0 ? d.dtb / 2.0 : d.dtb;
    io.beta = T(0.0);
  } else {
    dt = st == 0 ? d.dtb / 3.0 : (st == 1 ? d.dtb / 2.0 : d.dtb);
    io.beta = T(1.0);
  }
  io.dt = (T)dt;
  io.stored_halo = (step == 0 && st == 0) ? 1 : 0;
  io.last = st == nst - 1 ? 1 : 0;
  return io;
}

// Shared-memory copies of the current tile's member record, geometry and
// stage pointers; the tile code reads them like kernel parameters.
template <typename T>
struct TileCtx {
  MemberDesc<T> d;
  Geo<T> g;
  StageIO<T> io;
  int k;  // member whose record and geometry are loaded (-1: none)
};

// Point ctx at member k, stage (step, st).  Called by every thread between
// barriers; warp 0 alone does the work: when the member changes it copies the
// member record and then its geometry with coalesced word loads (two round
// trips), and lane 0 derives the stage pointers from the copy.
template <typename T>
__device__ __forceinline__ void ctx_load(TileCtx<T>& ctx, const BatchArgs<T>& a, int k, int step, int st) {
  __syncthreads();  // the previous tile is done with ctx
  if (threadIdx.x < 32) {
    if (ctx.k != k) {
      const int* src = reinterpret_cast<const int*>(a.mem + k);
      int* dst = reinterpret_cast<int*>(&ctx.d);
      for (int w = threadIdx.x; w < (int)(sizeof(MemberDesc<T>) / sizeof(int)); w += 32) dst[w] = __ldg(src + w);
      __syncwarp();
      const int* gsrc = reinterpret_cast<const int*>(a.geos + ctx.d.geo);
      int* gdst = reinterpret_cast<int*>(&ctx.g);
      for (int w = threadIdx.x; w < (int)(sizeof(Geo<T>) / sizeof(int)); w += 32) gdst[w] = __ldg(gsrc + w);
      __syncwarp();
    }
    if (threadIdx.x == 0) ctx.io = member_stage(ctx.d, a.rk, step, st);
  }
  __syncthreads();
  ctx.k = k;
}

template <typename T>
__device__ __forceinline__ int active_members(const BatchArgs<T>& a, int act, int step) {
  while (act > 0 && a.mem[act - 1].nbb <= step) --act;
  return act;
}

// Resident CTAs per SM of the batched phase kernels: their member geometry and
// stage pointers live in shared memory, so the pointers occupy registers; 3
// CTAs (85 registers) measured faster than 4 (spills) or 2 (occupancy).
constexpr int kBatchPhaseBlocks = 3;

// Tile phase of every active member (one launch per phase): blockIdx.x is the
// tile in the member-major tile list.  FP: the full-interior-tile path
// compiled in (launches of more than one wave), else the smaller edge-path-only
// code (launches whose CTAs all fit at once).
template <typename T, int TI, int TJ, bool UV, bool FP>
__global__ void __launch_bounds__(kTileThreads, kBatchPhaseBlocks) k_batch_phase(BatchArgs<T> a, int step, int st, int act) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ TileCtx<T> ctx;
  release_dependents();
  const int tile = blockIdx.x;
  __shared__ int s_k;
  if (threadIdx.x < 32) {
    const int k = member_of_warp(a.off.tile, act, tile);
    if (threadIdx.x == 0) s_k = k;
  }
  ctx.k = -1;
  __syncthreads();
  const int k = s_k;
  ctx_load(ctx, a, k, step, st);
  const Geo<T>& g = ctx.g;
  const TileBox b = tile_box_at(make_tiling_dev(TI, TJ, g.n), g.n, tile - __ldg(a.off.tile + k));
  T* sm = reinterpret_cast<T*>(smraw);
  if (!UV)
    tile_h<T, TI, TJ, FP>(g, ctx.io, b, sm);
  else
    tile_uv<T, TI, TJ, FP>(g, ctx.io, b, sm);
}

// End of a round: halo fill of every member's output and, for members with
// diagnostics, of the last stage input; then (second kernel) the diagnostics.
template <typename T>
__device__ __forceinline__ void batch_fill_item(const BatchArgs<T>& a, int item) {
  const int nf = __ldg(a.off.fill + a.count);
  if (item < nf) {
    const int k = member_of(a.off.fill, a.count, item);
    const MemberDesc<T>& d = a.mem[k];
    fill_halo_cell(a.geos[d.geo], d.x[0], d.x[1], d.x[2], item - __ldg(a.off.fill + k));
    return;
  }
  item -= nf;
  if (item < __ldg(a.off.lfill + a.count)) {
    const int k = member_of(a.off.lfill, a.count, item);
    const MemberDesc<T>& d = a.mem[k];
    T* const* L = a.rk == 2 ? d.y : d.z;
    fill_halo_cell(a.geos[d.geo], L[0], L[1], L[2], item - __ldg(a.off.lfill + k));
  }
}

template <typename T>
__device__ __forceinline__ void batch_diag_item(const BatchArgs<T>& a, int item) {
  const int k = member_of(a.off.diag, a.count, item);
  const MemberDesc<T>& d = a.mem[k];
  const Geo<T>& g = a.geos[d.geo];
  const int r = item - __ldg(a.off.diag + k);
  const int m = g.m;
  const int f = r / (m * m);
  const int c = r - f * m * m;
  T* const* L = a.rk == 2 ? d.y : d.z;
  DiagOut<T> o;
  T** op = reinterpret_cast<T**>(&o);
  for (int q = 0; q < 10; ++q) op[q] = d.diag[q];
  diag_cell(g, L[0], L[1], L[2], o, f, c / m, c % m);
}

template <typename T>
__global__ void __launch_bounds__(kTileThreads) k_batch_fill(BatchArgs<T> a) {
  wait_prior_grid();
  release_dependents();
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item < __ldg(a.off.fill + a.count) + __ldg(a.off.lfill + a.count)) batch_fill_item(a, item);
}

template <typename T>
__global__ void __launch_bounds__(kTileThreads) k_batch_diag(BatchArgs<T> a) {
  wait_prior_grid();
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item < __ldg(a.off.diag + a.count)) batch_diag_item(a, item);
}

// A whole batched round in one cooperative launch.  Each CTA walks its tiles
// of a phase (tile = blockIdx.x + k * gridDim.x over the active prefix), then
// all CTAs meet at a grid barrier; after the last phase the halo fills and
// diagnostics run as two more barrier-separated sweeps.
template <typename T, int TI, int TJ>
__global__ void __launch_bounds__(kTileThreads, 2) k_batch_round(BatchArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ TileCtx<T> ctx;
  T* sm = reinterpret_cast<T*>(smraw);
  const int nst = a.rk == 2 ? 2 : 3;
  const int nphase = a.max_nbb * nst * 2;
  unsigned gen = 0;
  int act = a.count;
  ctx.k = -1;
  for (int ph = 0; ph < nphase; ++ph) {
    const int step = ph / (2 * nst), st = (ph >> 1) % nst;
    const bool uv = ph & 1;
    act = active_members(a, act, step);
    const int ntiles = __ldg(a.off.tile + act);
    int k = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      while (__ldg(a.off.tile + k + 1) <= tile) ++k;
      ctx_load(ctx, a, k, step, st);
      const Geo<T>& g = ctx.g;
      const TileBox b = tile_box(make_tiling_dev(TI, TJ, g.n), g.n, tile - __ldg(a.off.tile + k));
      EdgeCnt cnt;
      int P;
      if (!uv) {
        Gather<T, TI, TJ, false> gat;
        tile_h_pro<T, TI, TJ>(g, ctx.io, b, sm, gat, cnt, P);
        tile_h_main<T, TI, TJ>(g, ctx.io, b, sm, gat, cnt, P);
      } else {
        Gather<T, TI, TJ, true> gat;
        tile_uv_pro<T, TI, TJ>(g, ctx.io, b, sm, gat, cnt, P);
        tile_uv_main<T, TI, TJ>(g, ctx.io, b, sm, gat, cnt, P);
      }
    }
    if (!grid_barrier(a.bar, gen, a.err, a.spin_limit)) {
      cp_async_wait_all();
      return;
    }
  }
  const int nfill = __ldg(a.off.fill + a.count) + __ldg(a.off.lfill + a.count);
  for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < nfill; item += gridDim.x * blockDim.x)
    batch_fill_item(a, item);
  if (!a.any_diag) return;
  if (!grid_barrier(a.bar, gen, a.err, a.spin_limit)) return;
  const int ndiag = __ldg(a.off.diag + a.count);
  for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < ndiag; item += gridDim.x * blockDim.x)
    batch_diag_item(a, item);
}

namespace {

template <typename T, int TI, int TJ, bool UV>
size_t batch_tile_smem() {
  using S = TileShape<TI, TJ>;
  return sizeof(T) * (UV ? S::kWordsUV : S::kWordsH) + sizeof(int) * kItemWords;
}

template <typename T, int TI, int TJ>
size_t batch_round_smem() {
  return std::max(batch_tile_smem<T, TI, TJ, false>(), batch_tile_smem<T, TI, TJ, true>());
}

// CTAs of one batched phase kernel (edge-only build) that fit on each device
// at once, recorded by prime_batch_tile (0 = not recorded).
constexpr int kMaxBatchDevices = 64;
template <typename T, int TI, int TJ, bool UV>
std::atomic<int>* batch_wave_slots() {  // relaxed: plans on several host threads may record them at once
  static std::atomic<int> slots[kMaxBatchDevices];
  return slots;
}

template <typename T, int TI, int TJ, bool UV>
cudaError_t prime_batch_phase() {
  cudaError_t e;
  for (auto k : {k_batch_phase<T, TI, TJ, UV, true>, k_batch_phase<T, TI, TJ, UV, false>})
    if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)batch_tile_smem<T, TI, TJ, UV>())) != cudaSuccess)
      return e;
  int dev, sms, per_sm;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxBatchDevices) return cudaSuccess;  // launches then keep the full-tile path
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_phase<T, TI, TJ, UV, false>, kTileThreads,
                                                         batch_tile_smem<T, TI, TJ, UV>())) != cudaSuccess)
    return e;
  batch_wave_slots<T, TI, TJ, UV>()[dev].store(sms * per_sm, std::memory_order_relaxed);
  return cudaSuccess;
}

template <typename T, int TI, int TJ>
cudaError_t prime_batch_tile() {
  cudaError_t e = prime_batch_phase<T, TI, TJ, false>();
  if (e != cudaSuccess) return e;
  if ((e = prime_batch_phase<T, TI, TJ, true>()) != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_batch_round<T, TI, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)batch_round_smem<T, TI, TJ>());
}

template <typename T, int TI, int TJ>
cudaError_t launch_batch_round_tile(BatchArgs<T> a, int max_tiles, int max_ctas, cudaStream_t s, int* grid_out) {
  const size_t smem = batch_round_smem<T, TI, TJ>();
  int dev, sms, per_sm;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_round<T, TI, TJ>, kTileThreads, smem)) !=
      cudaSuccess)
    return e;
  int grid = std::min(per_sm * sms, max_tiles);
  if (max_ctas > 0) grid = std::min(grid, max_ctas);
  if (grid < 1) return cudaErrorInvalidConfiguration;
  // the grid barrier counts arrivals in 31 bits: (phases + 2 end sweeps) x CTAs must stay below 2^31
  const long long arrivals = ((long long)a.max_nbb * (a.rk == 2 ? 2 : 3) * 2 + 2) * grid;
  if (arrivals >= (1ll << 31)) return cudaErrorInvalidValue;
  if (grid_out) *grid_out = grid;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)k_batch_round<T, TI, TJ>, dim3(grid), dim3(kTileThreads), args,
                                     smem, s);
}

template <typename T, int TI, int TJ, bool UV>
cudaError_t launch_batch_phase_tile(const BatchArgs<T>& a, int step, int st, int act, int ntiles, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ntiles);
  cfg.blockDim = dim3(kTileThreads);
  cfg.dynamicSmemBytes = batch_tile_smem<T, TI, TJ, UV>();
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int dev = -1;
  const int slots = (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxBatchDevices)
                        ? batch_wave_slots<T, TI, TJ, UV>()[dev].load(std::memory_order_relaxed) : 0;
  const bool one_wave = slots > 0 && ntiles <= slots;
  return one_wave ? cudaLaunchKernelEx(&cfg, k_batch_phase<T, TI, TJ, UV, false>, a, step, st, act)
                  : cudaLaunchKernelEx(&cfg, k_batch_phase<T, TI, TJ, UV, true>, a, step, st, act);
}

template <typename T, bool UV>
cudaError_t batch_phase_dispatch(const BatchArgs<T>& a, TileCfg c, int step, int st, int act, int ntiles,
                                 cudaStream_t s) {
  if (c.ti == 7 && c.tj == 32) return launch_batch_phase_tile<T, 7, 32, UV>(a, step, st, act, ntiles, s);
  if (c.ti == 8 && c.tj == 32) return launch_batch_phase_tile<T, 8, 32, UV>(a, step, st, act, ntiles, s);
  if (c.ti == 15 && c.tj == 32) return launch_batch_phase_tile<T, 15, 32, UV>(a, step, st, act, ntiles, s);
  if (c.ti == 16 && c.tj == 32) return launch_batch_phase_tile<T, 16, 32, UV>(a, step, st, act, ntiles, s);
  if (c.ti == 8 && c.tj == 16) return launch_batch_phase_tile<T, 8, 16, UV>(a, step, st, act, ntiles, s);
  if (c.ti == 16 && c.tj == 16) return launch_batch_phase_tile<T, 16, 16, UV>(a, step, st, act, ntiles, s);
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_small(void (*kern)(BatchArgs<T>), const BatchArgs<T>& a, int items, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((items + kTileThreads - 1) / kTileThreads);
  cfg.blockDim = dim3(kTileThreads);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, a);
}

}  // namespace

template <typename T>
cudaError_t prime_batch() {
  cudaError_t e;
  if ((e = prime_batch_tile<T, 7, 32>()) != cudaSuccess) return e;
  if ((e = prime_batch_tile<T, 8, 32>()) != cudaSuccess) return e;
  if ((e = prime_batch_tile<T, 15, 32>()) != cudaSuccess) return e;
  if ((e = prime_batch_tile<T, 16, 32>()) != cudaSuccess) return e;
  if ((e = prime_batch_tile<T, 8, 16>()) != cudaSuccess) return e;
  return prime_batch_tile<T, 16, 16>();
}

template <typename T>
cudaError_t launch_batch_round(const BatchArgs<T>& a, TileCfg c, int max_tiles, int max_ctas, cudaStream_t s,
                               int* grid_out) {
  if (c.ti == 7 && c.tj == 32) return launch_batch_round_tile<T, 7, 32>(a, max_tiles, max_ctas, s, grid_out);
  if (c.ti == 8 && c.tj == 32) return launch_batch_round_tile<T, 8, 32>(a, max_tiles, max_ctas, s, grid_out);
  if (c.ti == 15 && c.tj == 32) return launch_batch_round_tile<T, 15, 32>(a, max_tiles, max_ctas, s, grid_out);
  if (c.ti == 16 && c.tj == 32) return launch_batch_round_tile<T, 16, 32>(a, max_tiles, max_ctas, s, grid_out);
  if (c.ti == 8 && c.tj == 16) return launch_batch_round_tile<T, 8, 16>(a, max_tiles, max_ctas, s, grid_out);
  if (c.ti == 16 && c.tj == 16) return launch_batch_round_tile<T, 16, 16>(a, max_tiles, max_ctas, s, grid_out);
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_batch_phase(const BatchArgs<T>& a, TileCfg c, bool uv, int step, int st, int act, int ntiles,
                               cudaStream_t s) {
  return uv ? batch_phase_dispatch<T, true>(a, c, step, st, act, ntiles, s)
            : batch_phase_dispatch<T, false>(a, c, step, st, act, ntiles, s);
}

template <typename T>
cudaError_t launch_batch_end(const BatchArgs<T>& a, int nfill, int ndiag, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (nfill > 0) e = launch_small<T>(k_batch_fill<T>, a, nfill, s);
  if (e == cudaSuccess && ndiag > 0) e = launch_small<T>(k_batch_diag<T>, a, ndiag, s);
  return e;
}

#define BT_BATCH_INSTANTIATE(T)                                                                             \
  template cudaError_t prime_batch<T>();                                                                    \
  template cudaError_t launch_batch_round<T>(const BatchArgs<T>&, TileCfg, int, int, cudaStream_t, int*);   \
  template cudaError_t launch_batch_phase<T>(const BatchArgs<T>&, TileCfg, bool, int, int, int, int,       \
                                             cudaStream_t);                                                 \
  template cudaError_t launch_batch_end<T>(const BatchArgs<T>&, int, int, cudaStream_t);

}  // namespace bt
