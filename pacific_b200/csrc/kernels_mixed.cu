// kernels_mixed.cu -- mixed-precision instantiation of the DEM step kernels:
// FP32 contact law, forces, velocities and contact memory; FP64 positions,
// quaternions and contact decisions.
#define GG_DEFINE_SHARED_KERNELS 1
#include "kernels.cuh"

namespace gg {
GG_INSTANTIATE(float)
}
