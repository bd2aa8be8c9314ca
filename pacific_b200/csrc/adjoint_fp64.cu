// adjoint_fp64.cu -- the differentiable run and its adjoint in plain FP64
// (compiled like kernels_fp64.cu, without FMA contraction).
#include "adjoint.cuh"

namespace gg {
AdjointEngine* make_adjoint_fp64(const ContextView& v, int checkpoint_every, std::string& err) {
  return make_adjoint_engine<double, 4>(v, checkpoint_every, err);
}
}  // namespace gg
