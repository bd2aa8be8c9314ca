// adjoint_api.cu -- C ABI of the differentiable run (include/grains_gpu.h,
// "gradients" section): a handle that owns the tape and checkpoints of one
// context's run and the engine of the context's precision.
#include <cstring>
#include <string>

#include "../../include/grains_gpu.h"
#include "adjoint.h"

using namespace gg;

struct grains_gpu_adjoint {
  grains_gpu_ctx* ctx = nullptr;
  AdjointEngine* engine = nullptr;
  std::string err;
};

extern "C" {

int grains_gpu_adjoint_create(grains_gpu_ctx* ctx, int32_t checkpoint_every, grains_gpu_adjoint** out) {
  if (!ctx || !out || checkpoint_every < 1) return GRAINS_GPU_INVALID_ARGUMENT;
  *out = nullptr;
  auto* a = new grains_gpu_adjoint();
  a->ctx = ctx;
  ContextView v;
  int rc = context_view(ctx, &v, a->err);
  if (!rc) {
    if (cudaSetDevice(v.device) != cudaSuccess) {
      a->err = "cudaSetDevice failed";
      rc = GRAINS_GPU_CUDA_ERROR;
    } else {
      a->engine = v.precision == GRAINS_GPU_FP64 ? make_adjoint_fp64(v, checkpoint_every, a->err)
                                                 : make_adjoint_mixed(v, checkpoint_every, a->err);
      if (!a->engine) rc = GRAINS_GPU_CUDA_ERROR;
    }
  }
  *out = a;  // returned even on failure, so that the message can be read
  return rc;
}

int grains_gpu_adjoint_destroy(grains_gpu_adjoint* a) {
  if (!a) return 0;
  delete a->engine;
  delete a;
  return 0;
}

int grains_gpu_adjoint_last_error(const grains_gpu_adjoint* a, char* buf, size_t len) {
  if (!a || !buf || len == 0) return GRAINS_GPU_INVALID_ARGUMENT;
  std::strncpy(buf, a->err.c_str(), len - 1);
  buf[len - 1] = 0;
  return 0;
}

int grains_gpu_adjoint_law_slots(const grains_gpu_adjoint* a, int32_t* n_slots) {
  if (!a || !a->engine || !n_slots) return GRAINS_GPU_INVALID_ARGUMENT;
  *n_slots = a->engine->n_law_slots();
  return 0;
}

int grains_gpu_adjoint_forward(grains_gpu_adjoint* a, int32_t n_steps, double dt, double* position,
                               double* velocity, double* omega) {
  if (!a || !a->engine) return GRAINS_GPU_INVALID_ARGUMENT;
  ContextView v;
  if (int rc = context_view(a->ctx, &v, a->err)) return rc;
  return a->engine->forward(v, n_steps, dt, position, velocity, omega, a->err);
}

int grains_gpu_adjoint_contact_signature(const grains_gpu_adjoint* a, uint64_t* signature, int64_t* n_contacts) {
  if (!a || !a->engine || !signature || !n_contacts) return GRAINS_GPU_INVALID_ARGUMENT;
  unsigned long long s = 0;
  long long n = 0;
  a->engine->signature(&s, &n);
  *signature = (uint64_t)s;
  *n_contacts = (int64_t)n;
  return 0;
}

int grains_gpu_adjoint_backward(grains_gpu_adjoint* a, const double* dl_dposition, const double* dl_dvelocity,
                                const double* dl_domega, double* grad_position, double* grad_velocity,
                                double* grad_omega, double* grad_laws, int32_t n_grad_laws) {
  if (!a || !a->engine || n_grad_laws < 0) return GRAINS_GPU_INVALID_ARGUMENT;
  return a->engine->backward(dl_dposition, dl_dvelocity, dl_domega, grad_position, grad_velocity, grad_omega,
                             grad_laws, n_grad_laws, a->err);
}

}  // extern "C"
