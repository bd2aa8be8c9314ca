// noalloc.cu -- contact detection for spheres that allocates no memory.
//
// grains_gpu_sphere_contacts_noalloc is the allocation-free variant of the
// contact-list broadphase (contacts_kernel in kernels.cuh): it bins the
// spheres into the linked-cell grid, sorts them by cell and lists every pair
// whose overlap distance |x_j - x_i| - (r_i + r_j) is negative, with the same
// double-precision rounding as the context-based path.  All of its scratch
// (cell counts and ranges, the cell-sorted copy of the spheres) lives in the
// file-scope device array below, sized for at most kMaxSpheres spheres and
// kMaxCells cells; the caller passes only its inputs and outputs.
//
// It exists for callers that cannot call cudaMalloc: code running inside a
// stream capture that must not allocate, real-time loops where cudaMalloc's
// implicit device synchronisation is not acceptable, and hosts (a fluid solver
// coupling, a memory-budgeted service) that own every byte of device memory
// through their own pool.  The array takes sizeof(NoallocScratch) =
// 4,980,752 bytes (about 5.0 MB) on every GPU that loads the library, for as
// long as the process lives.
//
// Only the SET of output pairs is defined: the slot of each pair comes from an
// atomic counter, and the order of spheres inside a cell from atomic ranks, so
// the order of the pairs changes from call to call.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/grains_gpu.h"
#include "common.cuh"
#include "sphere_contact.cuh"

namespace {

constexpr int kMaxSpheres = 1 << 16;   // 65,536 spheres
constexpr int kMaxCells = 1 << 18;     // 262,144 cells
constexpr int kScanThreads = 1024;

struct NoallocScratch {
  int cell_count[kMaxCells];
  int cell_start[kMaxCells + 1];
  unsigned key[kMaxSpheres];
  unsigned rank[kMaxSpheres];
  int perm[kMaxSpheres];        // sorted slot -> input index
  double4 sorted[kMaxSpheres];  // (x, y, z, r) in cell order
};
static_assert(sizeof(NoallocScratch) == 4980752, "documented scratch size");

// Shared by every call on a device; keeps the last call's contents.
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

struct Grid {
  double ox, oy, oz, ex, ey, ez;
  int nbi, nbj, nbk;
};

__device__ __forceinline__ bool grid_cell(const Grid& g, double x, double y, double z, int& i, int& j, int& k) {
  i = int(floor(gg::xdiv(gg::xsub(x, g.ox), g.ex)));
  j = int(floor(gg::xdiv(gg::xsub(y, g.oy), g.ey)));
  k = int(floor(gg::xdiv(gg::xsub(z, g.oz), g.ez)));
  const bool ok = -1 < i && i < g.nbi && -1 < j && j < g.nbj && -1 < k && k < g.nbk;
  i = min(max(i, 0), g.nbi - 1);
  j = min(max(j, 0), g.nbj - 1);
  k = min(max(k, 0), g.nbk - 1);
  return ok;
}
__device__ __forceinline__ int grid_index(const Grid& g, int i, int j, int k) {
  return j * g.nbk * g.nbi + k * g.nbi + i;
}

// clears the counts of this call's cells and the caller's counter and status
__global__ void noalloc_clear(NoallocScratch* sc, int n_cells, unsigned long long* n_pairs, int* status) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n_cells) sc->cell_count[c] = 0;
  if (c == 0) {
    *n_pairs = 0ull;
    *status = 0;
  }
}

// Bins sphere s.  Only the 27 cells around a sphere are searched, which finds
// every contact when no two touching spheres are more than one cell apart,
// i.e. when the smallest cell edge is at least the largest diameter: a sphere
// whose diameter exceeds it sets GRAINS_GPU_CELL_TOO_SMALL.
__global__ void noalloc_bin(NoallocScratch* sc, Grid g, int n, const double* pos, const double* radius,
                            int* status) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int i, j, k;
  if (!grid_cell(g, pos[3 * s], pos[3 * s + 1], pos[3 * s + 2], i, j, k)) atomicOr(status, GRAINS_GPU_OUT_OF_GRID);
  if (2. * radius[s] > fmin(g.ex, fmin(g.ey, g.ez))) atomicOr(status, GRAINS_GPU_CELL_TOO_SMALL);
  const unsigned key = (unsigned)grid_index(g, i, j, k);
  sc->key[s] = key;
  sc->rank[s] = (unsigned)atomicAdd(&sc->cell_count[key], 1);
}

// exclusive scan of the counts by one block: each thread owns a contiguous run
__global__ void __launch_bounds__(kScanThreads) noalloc_scan(NoallocScratch* sc, int n_cells) {
  __shared__ int part[kScanThreads];
  const int per = (n_cells + kScanThreads - 1) / kScanThreads;
  const int b = threadIdx.x * per, e = min(b + per, n_cells);
  int sum = 0;
  for (int c = b; c < e; ++c) sum += sc->cell_count[c];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < kScanThreads; off <<= 1) {
    int v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = threadIdx.x > 0 ? part[threadIdx.x - 1] : 0;
  for (int c = b; c < e; ++c) {
    sc->cell_start[c] = run;
    run += sc->cell_count[c];
  }
  if (threadIdx.x == kScanThreads - 1) sc->cell_start[n_cells] = part[kScanThreads - 1];
}

__global__ void noalloc_scatter(NoallocScratch* sc, int n, const double* pos, const double* radius, int* status) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int slot = sc->cell_start[sc->key[s]] + (int)sc->rank[s];
  if (slot < 0 || slot >= n) {
    atomicOr(status, GRAINS_GPU_CUDA_ERROR);
    return;
  }
  sc->perm[slot] = s;
  sc->sorted[slot] = make_double4(pos[3 * s], pos[3 * s + 1], pos[3 * s + 2], radius[s]);
}

// contact test over the 27 surrounding cells; each pair is emitted once by its
// lower input index
__global__ void __launch_bounds__(256) noalloc_contacts(NoallocScratch* sc, Grid g, int n, int* pairs,
                                                        long long cap, unsigned long long* n_pairs) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const double4 xi = sc->sorted[s];
  const int id = sc->perm[s];
  int ci, cj, ck;
  grid_cell(g, xi.x, xi.y, xi.z, ci, cj, ck);
  const int i0 = max(ci - 1, 0), i1 = min(ci + 1, g.nbi - 1);
  for (int dj = -1; dj <= 1; ++dj) {
    const int j = cj + dj;
    if (j < 0 || j >= g.nbj) continue;
    for (int dk = -1; dk <= 1; ++dk) {
      const int k = ck + dk;
      if (k < 0 || k >= g.nbk) continue;
      const int t0 = sc->cell_start[grid_index(g, i0, j, k)];
      const int t1 = sc->cell_start[grid_index(g, i1, j, k) + 1];
      for (int t = t0; t < t1; ++t) {
        const int jd = sc->perm[t];
        if (!(id < jd)) continue;
        const double4 xj = sc->sorted[t];
        gg::D3 ab;
        double nab;
        const double dist =
            gg::sphere_sphere_overlap(gg::d3(xi.x, xi.y, xi.z), xi.w, gg::d3(xj.x, xj.y, xj.z), xj.w, &ab, &nab);
        if (dist < 0.) {
          const unsigned long long q = atomicAdd(n_pairs, 1ull);
          if ((long long)q < cap) {
            pairs[2 * q] = id;
            pairs[2 * q + 1] = jd;
          }
        }
      }
    }
  }
}

// Device address of the scratch, per device.  It is looked up again on every
// call whose stream is not being captured (the lookup is cheap then), so a new
// primary context after a cudaDeviceReset gets its own address; a call inside
// a stream capture uses the address of the last call outside one.
std::mutex g_addr_mutex;
NoallocScratch* g_addr[128] = {nullptr};

int scratch_address(int device, cudaStream_t st, NoallocScratch** out) {
  if (device < 0 || device >= 128) return GRAINS_GPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusActive;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();  // treat an unanswered query as a capture
    cap = cudaStreamCaptureStatusActive;
  }
  if (cap == cudaStreamCaptureStatusNone || !g_addr[device]) {
    if (cap != cudaStreamCaptureStatusNone) return GRAINS_GPU_NOT_READY;  // first call inside a capture
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return GRAINS_GPU_CUDA_ERROR;
    g_addr[device] = (NoallocScratch*)p;
  }
  *out = g_addr[device];
  return 0;
}

}  // namespace

extern "C" int grains_gpu_sphere_contacts_noalloc(int32_t n, const double* position, const double* radius,
                                                  const double origin[3], const double size[3], double cell_size,
                                                  int32_t* pairs, int64_t cap, int64_t* n_pairs, int32_t* status,
                                                  void* stream) {
  if (n < 0 || n > kMaxSpheres) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!origin || !size || !n_pairs || !status || (n > 0 && (!position || !radius)) || (cap > 0 && !pairs))
    return GRAINS_GPU_INVALID_ARGUMENT;
  Grid g;
  g.ox = origin[0];
  g.oy = origin[1];
  g.oz = origin[2];
  // the linked-cell grid of LinkedCell::set (LinkedCell.cpp:69-98); the cell
  // counts are checked as doubles before any conversion to int
  if (!(cell_size >= 0.) || !std::isfinite(cell_size)) return GRAINS_GPU_INVALID_ARGUMENT;
  double ext[3];
  int nb[3];
  for (int a = 0; a < 3; ++a) {
    if (!(size[a] > 0.) || !std::isfinite(size[a]) || !std::isfinite(origin[a])) return GRAINS_GPU_INVALID_ARGUMENT;
    const double q = cell_size > gg::kEpsilon ? (size[a] + gg::kEpsilon) / cell_size : 1.;
    if (!(q < (double)kMaxCells + 1.)) return GRAINS_GPU_INVALID_ARGUMENT;
    nb[a] = (int)q;
    if (!nb[a]) nb[a] = 1;
    ext[a] = size[a] / nb[a];
  }
  const long long cells = (long long)nb[0] * nb[1] * nb[2];
  if (cells <= 0 || cells > kMaxCells) return GRAINS_GPU_INVALID_ARGUMENT;
  g.ex = ext[0];
  g.ey = ext[1];
  g.ez = ext[2];
  g.nbi = nb[0];
  g.nbj = nb[1];
  g.nbk = nb[2];
  const int n_cells = (int)cells;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return GRAINS_GPU_CUDA_ERROR;
  NoallocScratch* sc = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  if (int rc = scratch_address(device, st, &sc)) return rc;
  unsigned long long* cnt = (unsigned long long*)n_pairs;
  noalloc_clear<<<(n_cells + 255) / 256, 256, 0, st>>>(sc, n_cells, cnt, status);
  if (cudaPeekAtLastError() != cudaSuccess) return GRAINS_GPU_CUDA_ERROR;
  if (n > 0) {
    noalloc_bin<<<(n + 255) / 256, 256, 0, st>>>(sc, g, n, position, radius, status);
    noalloc_scan<<<1, kScanThreads, 0, st>>>(sc, n_cells);
    noalloc_scatter<<<(n + 255) / 256, 256, 0, st>>>(sc, n, position, radius, status);
    noalloc_contacts<<<(n + 255) / 256, 256, 0, st>>>(sc, g, n, pairs, (long long)cap, cnt);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : GRAINS_GPU_CUDA_ERROR;
}

