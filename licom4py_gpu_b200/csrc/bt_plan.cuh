// bt_plan.cuh - the plan object behind bt_plan_t (host side, internal to libbt.so).
//
// A plan holds one resolution's geometry (the caller's constant arrays and
// the halo gather tables built from them), the member scratch of the
// single-integration entry points, launch options and the graph cache.

#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "bt_launch.cuh"
#include "licom_bt.h"

using namespace bt;

// The kernels read the 2x2 matrix arrays (a_c2l, a_l2c, a_gct: four values
// per cell) with 16-byte copies and vector loads, so each must start on a
// 16-byte boundary.
inline bool matrices_aligned(const bt_grid_desc* d) {
  return (((uintptr_t)d->a_c2l | (uintptr_t)d->a_l2c | (uintptr_t)d->a_gct) & 15) == 0;
}

struct bt_plan;
namespace bt {
// Build the tile constant blocks of plan p for tile shape t if it has none (bt_capi.cu).
int ensure_const_blocks_any(bt_plan* p, TileCfg t, cudaStream_t s);
}  // namespace bt

struct bt_plan {
  int n = 0, m = 0, nh = 0, dtype = BT_F64, device = 0;
  TileCfg tile{8, 32};
  int mode = BT_MODE_STREAM;
  const void* c[17] = {};
  int route[24] = {};
  void* d_hsrc = nullptr;  // int2[6*nh]
  void* d_hw = nullptr;    // T[6*nh*2]
  void* scratch = nullptr; // Y (3 fields) + Y2 (3 fields) + edge lines
  size_t field_elems = 0;
  cudaStream_t cap_stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // graph cache
  cudaGraphExec_t gexec = nullptr;
  std::vector<uintptr_t> gkey;
  // tile constant blocks, one buffer per tile shape used (built on first use, see ensure_const_blocks):
  // the plan's own rounds use the plan's tile, batched rounds the batch's
  struct ConstBlocks {
    TileCfg tile{0, 0};
    void* ptr = nullptr;
  };
  ConstBlocks cblks[6];
  const ConstBlocks* cblk_for(TileCfg t) const {
    for (const ConstBlocks& c : cblks)
      if (c.ptr && c.tile.ti == t.ti && c.tile.tj == t.tj) return &c;
    return nullptr;
  }
  // host copy of the halo gather sources (the resident mode's dependency lists are built from it)
  std::vector<int2> h_src;
  // resident mode: dependency lists and progress flags of the tile shape res_tile, one device block:
  // dep_off [tiles + 1], dep_idx [ndep], flags [tiles], abort word
  TileCfg res_tile{0, 0};
  int* d_res = nullptr;
  int res_tiles = 0, res_ndep = 0;
  // persistent mode: barrier counter + device error flag, options
  unsigned* d_flags = nullptr;  // [0] barrier counter, [1] error bits
  int max_ctas = 0;
  long long spin_limit = 1ll << 24;
  int full_tiles = -1;  // BT_OPT_FULL_TILES
  int last_grid = 0;
  // optional kernel timing: event pairs on the launch stream around the round
  // kernel (persistent mode) or each phase kernel (stream mode), with their kind
  int timing = 0;
  mutable std::vector<cudaEvent_t> tev;
  mutable std::vector<int> tkind;
  mutable size_t tev_used = 0;

  // Record the start event of a timed kernel of the given kind (nullptr if timing is off).
  cudaError_t time_begin(int kind, cudaStream_t s, cudaEvent_t* stop) const {
    *stop = nullptr;
    if (!timing) return cudaSuccess;
    if (tev_used + 2 > tev.size()) {
      for (int k = 0; k < 2; ++k) {
        cudaEvent_t ev;
        cudaError_t e = cudaEventCreate(&ev);
        if (e != cudaSuccess) return e;
        tev.push_back(ev);
      }
    }
    tkind.resize(tev.size() / 2);
    tkind[tev_used / 2] = kind;
    cudaEvent_t start = tev[tev_used];
    *stop = tev[tev_used + 1];
    tev_used += 2;
    return cudaEventRecord(start, s);
  }

  size_t esize() const { return dtype == BT_F64 ? 8 : 4; }
  // scratch layout: 6 stage fields, edge lines (24 n), then on a 256-byte boundary (16-byte copies)
  // the face cache blocks, sized for every tile shape
  size_t face_offset() const { return ((6 * field_elems + 24 * (size_t)n) * esize() + 255) & ~(size_t)255; }
  size_t scratch_bytes() const { return face_offset() + face_cache_elems(n) * esize(); }
  void* scratch_field(int k) const { return (char*)scratch + (size_t)k * field_elems * esize(); }
  void* edge_lines() const { return scratch_field(6); }
  void* face_x() const { return (char*)scratch + face_offset(); }

  // geometry for kernels of tile shape t (its constant blocks if built)
  template <typename T>
  Geo<T> geo_tile(TileCfg t) const {
    Geo<T> g = geo_arrays<T>();
    const ConstBlocks* c = cblk_for(t);
    g.cblk = c ? (const T*)c->ptr : nullptr;
    g.cblk_ti = c ? t.ti : 0;
    g.cblk_tj = c ? t.tj : 0;
    return g;
  }
  template <typename T>
  Geo<T> geo() const {
    return geo_tile<T>(tile);
  }
  // geometry without constant blocks (the arrays only)
  template <typename T>
  Geo<T> geo_arrays() const {
    Geo<T> g;
    g.n = n;
    g.m = m;
    g.nh = nh;
    g.dzph_x = (const T*)c[0];
    g.dzph_y = (const T*)c[1];
    g.rdx = (const T*)c[2];
    g.rdy = (const T*)c[3];
    g.a_f = (const T*)c[4];
    g.c2l = (const T*)c[8];
    g.l2c = (const T*)c[9];
    g.gct = (const T*)c[12];
    g.sina = (const T*)c[13];
    g.rda = (const T*)c[14];
    g.c_dy = (const T*)c[15];
    g.d_dx = (const T*)c[16];
    g.hsrc = (const int2*)d_hsrc;
    g.hw = (const T*)d_hw;
    g.cblk = nullptr;
    g.cblk_ti = g.cblk_tj = 0;
    std::memcpy(g.route, route, sizeof(route));
    return g;
  }
};
