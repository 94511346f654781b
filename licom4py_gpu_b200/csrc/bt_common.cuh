// bt_common.cuh - shared types of the barotropic duogrid solver (device + host).
//
// One "member" is one barotropic integration: six cubed-sphere faces of
// N x N cells, stored like the reference as (6, M, M) arrays, M = N + 6
// (3-cell halo per side), row-major, axis -2 = Fortran i ("x"), axis -1 =
// Fortran j ("y").  All six faces of a member live on one GPU.
//
// Halo cells are never exchanged between devices.  During a round they are
// not materialised at all: a kernel that needs a halo value computes it from
// the neighbouring face's interior through a precomputed gather table
// (two source cells and two linear-interpolation weights per halo cell, the
// composition of the reference's halo copy and kinked->extended remap), and
// for vectors through the c2l/l2c rotations.  Halos are written out only at
// the end of a round, for the returned state.

#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bt {

constexpr int kHalo = 3;
enum Side { kE = 0, kW = 1, kN = 2, kS = 3 };  // communication.py:32

// Linear offset of cell (i, j) of face f in a member's (6, M, M) field.
__host__ __device__ __forceinline__ long cell(int f, int i, int j, int m) {
  return ((long)f * m + i) * m + j;
}

// Number of halo cells per face and the id of halo cell (i, j) in [0, nh).
// Order: rows 0..2 (all columns), rows M-3..M-1 (all columns), then the W
// band (rows 3..M-4, cols 0..2) and the E band (rows 3..M-4, cols M-3..M-1).
__host__ __device__ __forceinline__ int halo_count(int m) { return 12 * (m - 6) + 36; }

__host__ __device__ __forceinline__ bool is_interior(int i, int j, int m) {
  return i >= kHalo && i < m - kHalo && j >= kHalo && j < m - kHalo;
}

__host__ __device__ __forceinline__ int halo_id(int i, int j, int m) {
  if (i < kHalo) return i * m + j;
  if (i >= m - kHalo) return 3 * m + (i - (m - kHalo)) * m + j;
  const int n = m - 6;
  if (j < kHalo) return 6 * m + (i - kHalo) * 3 + j;
  return 6 * m + 3 * n + (i - kHalo) * 3 + (j - (m - kHalo));
}

// Routing entry for side d of face f: neighbour face, its side, reversed flag.
__host__ __device__ __forceinline__ int route_pack(int nb, int side, int rev) {
  return nb | (side << 4) | (rev << 6);
}
__host__ __device__ __forceinline__ int route_nb(int r) { return r & 15; }
__host__ __device__ __forceinline__ int route_side(int r) { return (r >> 4) & 3; }
__host__ __device__ __forceinline__ int route_rev(int r) { return (r >> 6) & 1; }

// Geometry of one resolution (shared by every member of that resolution).
template <typename T>
struct Geo {
  int n, m, nh;
  const T* dzph_x;  // (6,M,M)
  const T* dzph_y;
  const T* rdx;
  const T* rdy;
  const T* a_f;
  const T* c2l;     // (6,M,M,2,2)
  const T* l2c;     // (6,M,M,2,2)
  const T* gct;     // (6,M,M,2,2)
  const T* sina;
  const T* rda;
  const T* c_dy;
  const T* d_dx;
  const int2* hsrc; // (6, nh) source offsets (absolute within the member)
  const T* hw;      // (6, nh, 2) interpolation weights
  // Tile constant blocks for tiles of cblk_ti x cblk_tj cells (TileShape::cW words
  // per tile): the image of phase UV's shared-memory constant area
  // (TileShape::uG .. uCEnd), then the depths of the tile's x and y faces; phase
  // H of full interior tiles assembles its constants from its own block and its
  // four neighbours'.  nullptr, or another tile shape: the arrays above are read.
  const T* cblk;
  int cblk_ti, cblk_tj;
  int route[24];    // f*4 + side
};

// Pointers of one RK stage of one member.
template <typename T>
struct StageIO {
  const T* h;   // stage input (stencil reads)
  const T* u;
  const T* v;
  const T* hp;  // RK base (pointwise reads)
  const T* up;
  const T* vp;
  T* h_out;     // stage outputs (interior cells only)
  T* u_out;
  T* v_out;
  T* fx;        // face cache, one block per tile (bt_stencil.cuh, TileShape::fW): for every x face
                // and y face of the tile its averaged normal velocity, viscous correction and
                // celerity flux, written by phase H, read by phase UV of the same tile
  T dt;
  T beta;
  int stored_halo;  // 1: the inputs' halo cells hold valid values (first stage of a round)
  int last;         // 1: last stage of the substep (mass-flux edge average active)
};

// Error bits a kernel can raise in the plan's device flag.
enum DeviceError { kErrBarrierTimeout = 1, kErrNeighbourTimeout = 2 };

// Everything one persistent launch needs to run a whole round of one member.
template <typename T>
struct RoundArgs;

// Tile decomposition of the N x N interior of each face.
struct Tiling {
  int ti, tj;        // tile extent (rows, cols)
  int nti, ntj;      // tiles per face along i and j
  __host__ __device__ int tiles_per_face() const { return nti * ntj; }
};

// Neighbour synchronisation of the tile-resident round kernel (bt_resident.cuh).
// Each tile's flag has a 128-byte line of its own (kResFlagStride ints): the
// flags are polled continuously, and packing them would send every poll of
// the grid to a handful of L2 lines.
constexpr int kResFlagStride = 32;
struct ResSync {
  const int* dep_off;  // (tiles + 1) offsets into dep_idx
  const int* dep_idx;  // the tiles each tile waits for (symmetric relation)
  int* flags;          // tile t's flag at flags[t * kResFlagStride]: phases completed in this launch
  int* abort;          // set by a tile whose wait gave up; ends every other wait
};

template <typename T>
struct RoundArgs {
  Geo<T> g;
  Tiling t;
  const T* x0[3];  // round input h0, ub, vb (halos valid)
  const T* b0[3];  // round input base h0p, ubp, vbp
  T* x[3];         // output / running state
  T* y[3];         // stage scratch
  T* z[3];         // second stage scratch (RK3)
  T* fx;           // face cache blocks (phase H -> phase UV)
  int nbb, rk;      // substeps of this launch, RK order
  int step0;        // substep index of the launch's first substep within the round (0: reads x0/b0)
  double dtb;
  unsigned* bar;   // grid barrier counter, zero at launch
  int* err;        // device error flag
  long long spin_limit;
};

}  // namespace bt
