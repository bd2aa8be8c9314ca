// adjoint.h -- host interface between the C ABI (adjoint_api.cu), the context
// (api.cu) and the per-precision adjoint engines (adjoint_fp64.cu,
// adjoint_mixed.cu).
#pragma once

#include <string>

#include <cuda_runtime.h>

#include "device_state.h"

struct grains_gpu_ctx;

namespace gg {

// What the adjoint engine reads of a context: set-up tables and the current
// particle arrays (any order; orig maps a slot to its upload index).
struct ContextView {
  int precision;
  int device;
  cudaStream_t stream;
  int n;
  int n_cells;
  int n_sys;
  int n_laws;
  int hist_cap;
  int spheres_only;     // every particle is a sphere
  int box_walls_only;   // every obstacle is a box
  int hooke_laws_only;  // every contact law is Hooke or HookeMemory
  int n_moving;
  const SysDev* sys;
  const ShapeDev* shapes;
  const ObstacleDev* obs;
  const int* cell_obs_start;
  const int* cell_obs_idx;
  const void* laws;
  const double4* xr;
  const double4* md;
  const int4* meta;
  const int* orig;
  const void* v;
  const void* w;
  const void* inertia;
};

// fills v from the context (api.cu); 0 or a GRAINS_GPU_* code with err set
int context_view(grains_gpu_ctx* c, ContextView* v, std::string& err);

class AdjointEngine {
 public:
  virtual ~AdjointEngine() {}
  // leapfrog run of n_steps from the context's current state; final state to
  // the host arrays (3n doubles each, upload order)
  virtual int forward(const ContextView& v, int n_steps, double dt, double* x, double* vel, double* w,
                      std::string& err) = 0;
  // adjoint of the last forward run
  virtual int backward(const double* gx, const double* gv, const double* gw, double* ox, double* ov, double* ow,
                       double* glaw, int n_glaw, std::string& err) = 0;
  virtual int n_law_slots() const = 0;
  // xor of a hash of every contact (evaluation, owner, partner) of the last
  // forward run, and the number of contacts summed over its evaluations
  virtual void signature(unsigned long long* sig, long long* n_contacts) const = 0;
  virtual size_t device_bytes() const = 0;
};

AdjointEngine* make_adjoint_fp64(const ContextView& v, int checkpoint_every, std::string& err);
AdjointEngine* make_adjoint_mixed(const ContextView& v, int checkpoint_every, std::string& err);

}  // namespace gg
