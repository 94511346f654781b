// bt_resident_f32.cu - float32 instantiation of the tile-resident round kernel
// (precision form, FMA contraction allowed as in bt_kernels_f32.cu).
#include "bt_resident.cuh"

namespace bt {
BT_INSTANTIATE_RESIDENT(float)
}  // namespace bt
