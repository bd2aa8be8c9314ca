// adjoint_mixed.cu -- the differentiable run and its adjoint in mixed
// precision: FP64 positions and contact decisions, FP32 velocities, contact
// law, memory and adjoint variables (parameter adjoints summed in FP64).
#include "adjoint.cuh"

namespace gg {
AdjointEngine* make_adjoint_mixed(const ContextView& v, int checkpoint_every, std::string& err) {
  return make_adjoint_engine<float, 4>(v, checkpoint_every, err);
}
}  // namespace gg
