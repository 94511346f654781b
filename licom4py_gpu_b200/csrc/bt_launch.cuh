// bt_launch.cuh - host-side launch interface of the barotropic kernels (internal C++).
#pragma once

#include <string>

#include "bt_common.cuh"
#include "bt_stencil.cuh"

namespace bt {

// Record the thread-local message returned by bt_last_error(); returns code.
int set_error(int code, const std::string& msg);

struct TileCfg {
  int ti, tj;
};

// Tile shapes compiled into the library (rows x columns of interior cells).
bool tile_cfg_supported(TileCfg c);
// Tile constant blocks (Geo::cblk) for tile shape c: elements needed, and a
// stream-ordered build from the constant arrays of g.
size_t const_block_elems(TileCfg c, int n);
template <typename T>
cudaError_t launch_const_blocks(const Geo<T>& g, TileCfg c, T* out, cudaStream_t s);
// Elements of the face cache blocks of one member at n cells per face edge,
// enough for every supported tile shape (the plan's tile can change later).
size_t face_cache_elems(int n);
Tiling make_tiling(TileCfg c, int n);

// Set kernel attributes (dynamic shared memory opt-in) for the current device.
template <typename T>
cudaError_t prime_kernels();
// Phase kernels of one stage.  full_tiles selects the kernel: 1 = the one with
// the full-interior-tile path, 0 = edge path only, -1 = by size (the edge-only
// kernel when the launch's CTAs all fit on the device at once).  Results are
// the same either way.
template <typename T>
cudaError_t launch_phase_h(const Geo<T>& g, const StageIO<T>& io, TileCfg cfg, cudaStream_t s, int full_tiles = -1);
// Which kernels those launches take at n: bit 0 set = phase H runs the full-tile
// kernel, bit 1 = phase UV (-1: unsupported tile shape).
template <typename T>
int phase_full_paths(TileCfg cfg, int n, int full_tiles);
template <typename T>
cudaError_t launch_phase_uv(const Geo<T>& g, const StageIO<T>& io, TileCfg cfg, cudaStream_t s, int full_tiles = -1);
// Persistent cooperative launch of a whole round (phases of all substeps);
// max_ctas > 0 caps the grid.  The grid size used is returned in *grid_out.
template <typename T>
cudaError_t launch_round(const RoundArgs<T>& a, TileCfg cfg, int max_ctas, cudaStream_t s, int* grid_out);
// Tile-resident round (one CTA per tile, neighbour flags; bt_resident.cuh).
bool resident_tile_supported(TileCfg c);
template <typename T>
cudaError_t prime_resident();
// CTAs of the resident kernel for tile shape c that fit on the current device at once.
template <typename T>
cudaError_t resident_capacity(TileCfg c, int* ctas);
template <typename T>
cudaError_t launch_resident(const RoundArgs<T>& a, const ResSync& rs, TileCfg cfg, cudaStream_t s);
// Materialise the halo cells of h (scalar) and/or (u, v) (vector) from their interiors.
template <typename T>
cudaError_t launch_fill_halo(const Geo<T>& g, T* h, T* u, T* v, cudaStream_t s);
template <typename T>
cudaError_t launch_diag(const Geo<T>& g, const T* h, const T* u, const T* v, const DiagOut<T>& d,
                        cudaStream_t s);

}  // namespace bt
