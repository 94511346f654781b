// bt_resident_f64.cu - float64 instantiation of the tile-resident round kernel.
// Built with -fmad=false like the other float64 kernels (bitwise equal results).
#define BT_DEFINE_COMMON
#include "bt_resident.cuh"

namespace bt {
BT_INSTANTIATE_RESIDENT(double)
}  // namespace bt
