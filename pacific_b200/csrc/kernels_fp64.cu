// kernels_fp64.cu -- plain FP64 instantiation of the DEM step kernels.
// Built with -fmad=false so that every double expression rounds like the
// reference's x86-64 build (no fused multiply-add contraction).
#include "kernels.cuh"

namespace gg {
GG_INSTANTIATE(double)
}
