// bt_kernels_f64.cu - float64 instantiation of the barotropic kernels (the drop-in path).
// Built with -fmad=false: no FMA contraction, so every float64 expression rounds
// like the reference's float64 arithmetic, operand by operand.
#define BT_DEFINE_COMMON
#include "bt_kernels.cuh"

namespace bt {
BT_INSTANTIATE(double)
}  // namespace bt
