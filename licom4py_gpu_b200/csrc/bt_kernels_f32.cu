// bt_kernels_f32.cu - float32 instantiation of the barotropic kernels (the precision form).
// FMA contraction is allowed here: the float32 form is checked against the
// float64 path by tolerance, not bit for bit.
#include "bt_kernels.cuh"

namespace bt {
BT_INSTANTIATE(float)
}  // namespace bt
