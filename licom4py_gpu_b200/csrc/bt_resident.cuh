// bt_resident.cuh - the tile-resident round kernel (BT_MODE_RESIDENT).
//
// The reference runs a round as one XLA while loop of nbb substeps
// (src/licom/momentum/barotr.py:41-87, lax.fori_loop at :61).  For grids whose
// tiles all fit on the GPU at once (C48, C96), this kernel runs the whole
// round in one cooperative launch with ONE CTA PER TILE, and each CTA keeps
// everything that does not change during the round on chip:
//
//   * the tile's constants of both phases (metric, depths, spacings) are
//     staged into shared memory once, at launch;
//   * phase H leaves the face cache (edge-averaged normal velocity, its
//     viscous correction and the celerity flux of every face of the tile) and
//     the raw velocities of the stencil region in phase UV's shared-memory
//     layout, so phase UV reads only the new h of its region from memory.
//
// Tiles synchronise with their neighbours only: after each phase a CTA
// publishes the number of phases it has completed (release store of its own
// flag), and before a phase it waits until every tile it depends on has
// completed the previous phase.  The dependency list of a tile (built on the
// host, bt_resident_deps) holds every tile owning a cell the tile reads in
// either phase -- its 3-cell stencil region, halo cells resolved to their
// gather sources, the neighbour face's 6-point lines along the face edges it
// touches -- and is made symmetric, so a tile is never more than one phase
// ahead of a tile it reads from or that reads from it: no buffer is
// overwritten while a neighbour may still read it.  Every wait is bounded by
// the plan's spin limit; a tile that gives up raises kErrNeighbourTimeout and
// an abort word that ends every other tile's wait, and all CTAs return.
//
// The arithmetic is the tile phases' own (bt_stencil.cuh, RES = true), so the
// results are bitwise identical to the stream, graph and persistent modes.

#pragma once

#include "bt_launch.cuh"

namespace bt {

// Resident CTAs per SM the kernel is compiled for (register cap 65536 / (256 *
// blocks)).  The float64 layouts of the larger tiles (16 x 16, 8 x 32: over
// 100 KB) fit only two CTAs per SM anyway, so they get the registers of two.
template <typename T, int TI, int TJ>
struct ResBlocks {
  static constexpr int value = (sizeof(T) == 8 && TI * TJ > 128) ? 2 : 3;
};

// Shared-memory layout of a resident CTA (words of T): phase H layout, phase
// H face fluxes, phase UV layout, then the gather item scratch (ints).
template <typename T, int TI, int TJ>
struct ResLayout {
  using S = TileShape<TI, TJ>;
  static constexpr int kPQ = up4(S::kWordsH);
  static constexpr int kUV = up4(kPQ + S::FX + S::FY);
  static constexpr int kWords = up4(kUV + S::kWordsUV);
  static constexpr size_t kBytes = sizeof(T) * kWords + sizeof(int) * kItemWords;
};

// Publish that this CTA has completed ``phases`` phases: every thread's global
// stores are ordered before the flag by the barrier and the (cumulative)
// release store.
__device__ __forceinline__ void res_publish(int* flag, int phases) {
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(flag), "r"(phases) : "memory");
}

// Wait until every dependency of ``tile`` has completed ``need`` phases.  The
// lanes of warp 0 poll one dependency each (relaxed loads, a fence after the
// last one), at most ``limit`` polls per dependency; the abort word is
// checked every 64 polls.  Returns false when the round must stop.
__device__ __forceinline__ bool res_wait(const ResSync& s, int tile, int need, int* err, long long limit) {
  __shared__ int s_ok;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const int b = s.dep_off[tile], e = s.dep_off[tile + 1];
    int ok = 1;
    for (int k = b + lane; k < e && ok; k += 32) {
      const int* fp = s.flags + s.dep_idx[k] * kResFlagStride;
      long long polls = 0;
      while (true) {
        int seen;
        asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(seen) : "l"(fp) : "memory");
        if (seen >= need) break;
        ++polls;
        if ((polls & 63) == 0) {
          int ab;
          asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(ab) : "l"(s.abort) : "memory");
          if (ab) {
            ok = 0;
            break;
          }
        }
        if (polls > limit) {
          atomicOr(err, kErrNeighbourTimeout);
          atomicExch(s.abort, 1);
          ok = 0;
          break;
        }
      }
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Phase H then phase UV of one stage for a tile of kind FULL.
template <typename T, int TI, int TJ, bool FULL>
__device__ __forceinline__ bool res_stage(const RoundArgs<T>& a, const ResSync& rsy, const StageIO<T>& io,
                                          const TileBox& b, T* sm, const ResSm<T>& rs, int tile, int done) {
  {
    Gather<T, TI, TJ, false, true> gat;
    EdgeCnt cnt;
    int P;
    tile_desc<T, TI, TJ, FULL, false, true>(a.g, io, b, gat, cnt, P, rs.items);
    if (done > 0 && !res_wait(rsy, tile, done, a.err, a.spin_limit)) return false;
    tile_h_main_t<T, TI, TJ, FULL, true>(a.g, io, b, sm, gat, cnt, P, rs);
    res_publish(rsy.flags + tile * kResFlagStride, done + 1);
  }
  {
    Gather<T, TI, TJ, true, true> gat;
    EdgeCnt cnt;
    int P;
    tile_desc<T, TI, TJ, FULL, true, true>(a.g, io, b, gat, cnt, P, rs.items);
    if (!res_wait(rsy, tile, done + 1, a.err, a.spin_limit)) {
      cp_async_wait_all();
      return false;
    }
    tile_uv_main_t<T, TI, TJ, FULL, true>(a.g, io, b, rs.uv, gat, cnt, P, rs);  // phase UV's own layout
    res_publish(rsy.flags + tile * kResFlagStride, done + 2);
  }
  return true;
}

// One CTA per tile (face-major order); the grid is exactly the tile count.
template <typename T, int TI, int TJ>
__global__ void __launch_bounds__(kTileThreads, ResBlocks<T, TI, TJ>::value) k_resident(RoundArgs<T> a, ResSync rsy) {
  using RL = ResLayout<T, TI, TJ>;
  using S = TileShape<TI, TJ>;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ StageIO<T> s_io;
  T* const sm = reinterpret_cast<T*>(smraw);
  ResSm<T> rs;
  rs.uv = sm + RL::kUV;
  rs.pq = sm + RL::kPQ;
  rs.hs = sm + S::hH;
  rs.items = reinterpret_cast<int*>(sm + RL::kWords);
  const int tile = blockIdx.x;
  const TileBox b = tile_box_at(a.t, a.g.n, tile);
  const bool full = tile_full(b, a.g.m, TI, TJ);
  // the constants of both phases, once per round (awaited by the first phase's barrier)
  if (full) {
    tile_h_consts<T, TI, TJ, true>(a.g, b, sm);
    tile_uv_consts<T, TI, TJ, true>(a.g, b, rs.uv);
  } else {
    tile_h_consts<T, TI, TJ, false>(a.g, b, sm);
    tile_uv_consts<T, TI, TJ, false>(a.g, b, rs.uv);
  }
  const int nst = a.rk == 2 ? 2 : 3;
  const int nstage = a.nbb * nst;
  for (int sg = 0; sg < nstage; ++sg) {
    if (threadIdx.x == 0) s_io = round_stage(a, a.step0 + sg / nst, sg % nst);
    __syncthreads();
    const bool ok = full ? res_stage<T, TI, TJ, true>(a, rsy, s_io, b, sm, rs, tile, 2 * sg)
                         : res_stage<T, TI, TJ, false>(a, rsy, s_io, b, sm, rs, tile, 2 * sg);
    if (!ok) {
      cp_async_wait_all();  // no copy may be left in flight when the CTA leaves
      return;
    }
  }
}

}  // namespace bt

namespace bt {
namespace {

template <typename T, int TI, int TJ>
cudaError_t prime_resident_tile() {
  return cudaFuncSetAttribute(k_resident<T, TI, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)ResLayout<T, TI, TJ>::kBytes);
}

template <typename T, int TI, int TJ>
cudaError_t resident_capacity_tile(int* ctas) {
  int dev, sms, per_sm;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = prime_resident_tile<T, TI, TJ>()) != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resident<T, TI, TJ>, kTileThreads,
                                                    ResLayout<T, TI, TJ>::kBytes);
  if (e != cudaSuccess) return e;
  *ctas = per_sm * sms;
  return cudaSuccess;
}

template <typename T, int TI, int TJ>
cudaError_t launch_resident_tile(RoundArgs<T> a, ResSync rs, cudaStream_t s) {
  a.t = make_tiling({TI, TJ}, a.g.n);
  void* args[] = {&a, &rs};
  return cudaLaunchCooperativeKernel((const void*)k_resident<T, TI, TJ>, dim3(6 * a.t.tiles_per_face()),
                                     dim3(kTileThreads), args, ResLayout<T, TI, TJ>::kBytes, s);
}

}  // namespace

#ifdef BT_DEFINE_COMMON
bool resident_tile_supported(TileCfg c) {
  return (c.ti == 8 && c.tj == 16) || (c.ti == 16 && c.tj == 16) || (c.ti == 8 && c.tj == 32);
}
#endif

template <typename T>
cudaError_t prime_resident() {
  cudaError_t e = prime_resident_tile<T, 8, 16>();
  if (e == cudaSuccess) e = prime_resident_tile<T, 16, 16>();
  if (e == cudaSuccess) e = prime_resident_tile<T, 8, 32>();
  return e;
}

template <typename T>
cudaError_t resident_capacity(TileCfg c, int* ctas) {
  if (c.ti == 8 && c.tj == 16) return resident_capacity_tile<T, 8, 16>(ctas);
  if (c.ti == 16 && c.tj == 16) return resident_capacity_tile<T, 16, 16>(ctas);
  if (c.ti == 8 && c.tj == 32) return resident_capacity_tile<T, 8, 32>(ctas);
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_resident(const RoundArgs<T>& a, const ResSync& rs, TileCfg c, cudaStream_t s) {
  if (c.ti == 8 && c.tj == 16) return launch_resident_tile<T, 8, 16>(a, rs, s);
  if (c.ti == 16 && c.tj == 16) return launch_resident_tile<T, 16, 16>(a, rs, s);
  if (c.ti == 8 && c.tj == 32) return launch_resident_tile<T, 8, 32>(a, rs, s);
  return cudaErrorInvalidValue;
}

#define BT_INSTANTIATE_RESIDENT(T)                                                           \
  template cudaError_t prime_resident<T>();                                                  \
  template cudaError_t resident_capacity<T>(TileCfg, int*);                                  \
  template cudaError_t launch_resident<T>(const RoundArgs<T>&, const ResSync&, TileCfg, cudaStream_t);

}  // namespace bt
