// Batched-round kernels, float64 (compiled with -fmad=false: the arithmetic
// rounds like the single-member float64 kernels, term by term).
#include "bt_batch_kernels.cuh"

namespace bt {
BT_BATCH_INSTANTIATE(double)
}  // namespace bt
