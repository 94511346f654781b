// Batched-round kernels, float32 precision form (FMA contraction allowed, like
// the single-member float32 kernels).
#include "bt_batch_kernels.cuh"

namespace bt {
BT_BATCH_INSTANTIATE(float)
}  // namespace bt
