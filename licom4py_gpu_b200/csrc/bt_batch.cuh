// bt_batch.cuh - batched rounds: many independent integrations (ensemble
// members, served requests) of possibly different resolutions advanced
// together, in one persistent launch per round or one launch per phase.
//
// The tile work of a phase is the concatenation of every active member's
// tiles (all six faces of each).  Members are ordered by their substep count
// of the round, largest first, so the members still running at substep s
// always form a prefix of the list and their tiles a prefix of the tile
// space: a member that has done its substeps simply drops off the end
// ("retires") and the remaining phases get shorter.  Every tile uses the
// same TI x TJ shape; geometry is per resolution and shared by all members
// of that resolution.

#pragma once

#include "bt_launch.cuh"

namespace bt {

// One member of a batched round (device copy, written by the host per call).
template <typename T>
struct MemberDesc {
  const T* x0[3];  // round input h0, ub, vb (halo cells valid)
  const T* b0[3];  // round input base h0p, ubp, vbp
  T* x[3];         // output state (written by the last stage of each substep)
  T* y[3];         // stage scratch
  T* z[3];         // second stage scratch (RK3)
  T* fx;           // face cache blocks
  T* diag[10];     // STATE_KEYS[6:16] outputs, all null when not wanted
  double dtb;
  int geo;         // index into the call's geometry table
  int nbb;         // substeps of this round (non-increasing along the list)
};

// Prefix offsets of the member list (count + 1 entries each).
struct BatchOffsets {
  const int* tile;  // tiles of members [0, k)
  const int* fill;  // halo items of the output fill (6 nh per member)
  const int* lfill; // halo items of the last-stage-input fill (members with diagnostics)
  const int* diag;  // diagnostic cells (6 M^2 per member with diagnostics)
};

template <typename T>
struct BatchArgs {
  const Geo<T>* geos;
  const MemberDesc<T>* mem;
  BatchOffsets off;
  int count;
  int rk;
  int max_nbb;
  int any_diag;
  unsigned* bar;   // grid barrier counter, zero at launch (persistent launch)
  int* err;        // device error flag
  long long spin_limit;
};

// Host launchers (bt_batch_kernels.cuh, instantiated for double and float).
template <typename T>
cudaError_t prime_batch();
// One cooperative launch for the whole round; max_tiles = tiles of the first
// phase (all members), max_ctas > 0 caps the grid; the grid used is returned.
template <typename T>
cudaError_t launch_batch_round(const BatchArgs<T>& a, TileCfg c, int max_tiles, int max_ctas, cudaStream_t s,
                               int* grid_out);
// One phase (H or UV) of stage st of substep step over the first act members
// (ntiles tiles), launched with a programmatic dependency on the previous kernel.
template <typename T>
cudaError_t launch_batch_phase(const BatchArgs<T>& a, TileCfg c, bool uv, int step, int st, int act, int ntiles,
                               cudaStream_t s);
// Halo fills (nfill items) and diagnostics (ndiag cells, may be 0) after the last phase.
template <typename T>
cudaError_t launch_batch_end(const BatchArgs<T>& a, int nfill, int ndiag, cudaStream_t s);

}  // namespace bt
