// api.cu -- the C ABI of include/grains_gpu.h: context, device memory, set-up
// tables (shapes, domains, contact laws, obstacles, obstacle-cell links) and
// the orchestration of the DEM step kernels, with the step loop
// replayed from CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/grains_gpu.h"
#include "adjoint.h"
#include "device_state.h"
#include "format.cuh"
#include "io.h"
#include "gjk.cuh"
#include "sphere_contact.cuh"

using namespace gg;

namespace {

struct ShapeHost {
  int type = 0;
  std::vector<double> params;
  std::vector<double> verts;
  std::vector<std::vector<int>> faces;
  // vertex adjacency of a polyhedron (Polyhedron::m_cobound, built by
  // Polyhedron::BuildPolyhedron, Polyhedron.cpp:338-339): for every face, each
  // vertex lists the vertex that follows it on the face
  std::vector<int> adj_start, adj;
  double volume = 0, circ = 0;
  double inertia[3] = {0, 0, 0};
  double lext[3] = {0, 0, 0};
  D3 ext{0, 0, 0};
  double radius = 0, half_height = 0;
};

struct LawHost {
  int type = -1;
  double p[11] = {0};  // kn, en, etat, muc, kt, mur, etarpf, epst, kr, Es, Gs
  double beta = 0;
};

struct SysHost {
  bool has_domain = false;
  grains_gpu_domain dom{};
  int nbi = 1, nbj = 1, nbk = 1;
  double ex = 0, ey = 0, ez = 0;
  std::map<std::pair<int, int>, LawHost> laws;
  std::vector<grains_gpu_obstacle> obs;
  std::vector<grains_gpu_obstacle_loading> loads;  // explicit imposed motions
};

template <typename T>
T* dalloc(size_t n, std::vector<void*>& pool) {
  void* p = nullptr;
  if (n == 0) n = 1;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
  pool.push_back(p);
  return static_cast<T*>(p);
}

}  // namespace

struct grains_gpu_ctx {
  grains_gpu_config cfg{};
  int precision = GRAINS_GPU_MIXED;
  int hist_cap = 24;
  cudaStream_t stream = nullptr;
  std::string err;
  std::vector<ShapeHost> shapes;
  std::vector<SysHost> sys;
  // device memory
  std::vector<void*> pool;        // capacity-sized buffers (allocated at create)
  std::vector<void*> table_pool;  // tables rebuilt at upload
  size_t rsize = 4;               // sizeof(R)
  int64_t cap = 0;
  int64_t n = 0;
  int n_cells = 0;
  bool uploaded = false;
  bool tables_dirty = true;
  char* stage = nullptr;  // device staging of update / download in upload order (30 x 8 B per particle)
  char* row_scratch = nullptr;  // grains_gpu_update_particle_rows: rows, slot of every upload index
  int fluid_corrected = 0;      // grains_gpu_set_fluid
  // host copies of the uploaded particles for the fluid coupling's export
  // (upload order): id, shape, mass, principal inertia, circumscribed radius,
  // density (grains_gpu_set_fluid; else mass / volume)
  struct {
    std::vector<int> id, shape;
    std::vector<double> mass, inertia, radius, density;
  } fh;
  double* d_hydro = nullptr;    // grains_gpu_set_hydro_forces: 6 doubles per upload index
  bool hydro_on = false;
  bool sorted = false;      // cur arrays are in cell order for the current positions
  bool keys_valid = false;  // key and cell counts hold the cells of the current positions
  bool pending_kick2 = false;
  double pending_dt = 0;
  bool has_basis = false;    // a basis per particle is kept (non-spheres, or given at upload)
  bool all_spheres = true;   // every particle is a sphere
  bool has_convex = false;
  StepArgs<float> af{};
  StepArgs<double> ad{};
  // raw buffer pointers (two copies of particle arrays)
  struct Bufs {
    double4 *xr, *q;
    double* basis;
    void *v, *w, *wbf, *F, *T, *inertia;
    double4* md;
    int4* meta;
    int* orig;
    unsigned* key;  // cell key of the current positions
  } buf[2]{};
  int cur = 0;  // which copy is current
  void* hist[2] = {nullptr, nullptr};
  int* hist_n[2] = {nullptr, nullptr};
  int hcur = 0;  // hist[hcur] = latest memory (prev for the next force evaluation)
  int* coord = nullptr;
  int* perm = nullptr;
  int *cell_count = nullptr, *cell_start = nullptr, *cell_cursor = nullptr, *block_sums = nullptr;
  StatsDev* stats = nullptr;
  double* clock = nullptr;  // the reference's m_time, advanced by the obstacle moves
  int* clist = nullptr;   // contact lists (scratch of the force evaluation)
  int* ccount = nullptr;
  void* res_f = nullptr;  // per list entry: force and contact flag, torque (R4 each)
  void* res_t = nullptr;
  int4* work = nullptr;   // owned list entries of an evaluation
  int* work_n = nullptr;
  GjkOut* gjk_out = nullptr;  // per work item: the GJK kernel's narrowphase result (convex scenarios)
  int* gjk_next = nullptr;    // the GJK kernel's work-item counter
  int* gjk_order = nullptr;   // the GJK work items grouped by shape pair
  int* gjk_bins = nullptr;    // their bin counts and cursors
  int clist_cap = 0;
  int64_t clist_alloc = 0;
  int* pairs = nullptr;  // contact pairs of the last compute_forces (diagnostic)
  int pairs_cap = 0;
  unsigned long long* pairs_n = nullptr;
  double* pair_force = nullptr;  // force on the lower id of each diagnostic contact pair
  int* pair_sys = nullptr;       // system of each diagnostic contact pair
  int* cand = nullptr;   // candidate pairs (diagnostic, separate from the contact pairs)
  int cand_cap = 0;
  unsigned long long* cand_n = nullptr;
  // tables
  SysDev* d_sys = nullptr;
  ShapeDev* d_shapes = nullptr;
  double* d_verts = nullptr;
  int* d_adj_start = nullptr;  // polyhedron adjacency over the vertex table
  int* d_adj = nullptr;
  ObstacleDev* d_obs = nullptr;
  LoadingDev* d_loads = nullptr;
  int* d_load_flags = nullptr;  // per system: a loading active over this step, over the previous one
  // force-driven obstacles: partial contact forces (kForceBlocks x kMaxForceObstacles x 3) and the
  // controller history per system; null when no obstacle has an imposed force
  double* d_force_part = nullptr;
  double* d_force_pid = nullptr;
  int n_force_obs = 0;
  bool obs_force_valid = false;  // the list entries hold the results of a force evaluation
  int *d_cell_obs_start = nullptr, *d_cell_obs_idx = nullptr, *d_moving = nullptr;
  void* d_laws = nullptr;
  std::vector<SysDev> h_sys;
  std::vector<ObstacleDev> h_obs;
  int n_moving = 0;  // moving obstacles over all systems
  // graphs of two middle steps, by the starting (cur, hcur) buffer selection
  cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
  double graph_dt[4] = {0, 0, 0, 0};
  int64_t steps_done = 0;
  double gjk_tol = kEpsilon;  // GrainsExec::m_colDetTolerance
  int gjk_sv = 0;             // GrainsExec::m_colDetGJK_SV
  int gjk_accel = 0;          // GrainsExec::m_colDetAcceleration
  int gjk_history = 0;        // GrainsExec::m_colDetWithHistory
  GjkDir* gdir[2] = {nullptr, nullptr};  // collision histories, selected by hcur like the memory rows
  int* gdir_n[2] = {nullptr, nullptr};
  // launch and grid tuning (grains_gpu_set_tuning / grains_gpu_autotune)
  double cell_factor = 1.0;
  int contacts_block = 256;
  int forces_block = 128;
  int list_capacity = 0;  // 0: 32 slots for spheres, 64 when other shapes are present
  int gather_every = 16;  // steps between two gathers of the arrays into cell order
  int since_gather = 0;   // sorts without a gather since the last one
  int persistent = 0;     // middle steps in one cooperative launch instead of graphs
  long long barrier_polls = 1ll << 24;  // its grid-barrier wait bound (grains_gpu_set_barrier_test)
  int barrier_skip_block = -1;
  unsigned* pbar = nullptr;  // grid-barrier state of the persistent launch
  int* psums = nullptr;      // its scan scratch (one int per block)
  int pblocks = 0;
  // reload and RawData files (io.cu): particle names by upload index, sorted
  // (system, id) keys, obstacle ids, per-particle record attributes
  int* d_row_id = nullptr;
  int* d_row_sys = nullptr;
  unsigned long long* d_row_keys = nullptr;
  int* d_key_rows = nullptr;
  RecordAttr* d_attr = nullptr;
  int* d_obs_id = nullptr;
  int* d_sys_obs_offset = nullptr;
  int moved = 0;  // a move since the upload: transform types gain ROTATION | TRANSLATION
  IoScratch io;
};

namespace {

int fail(grains_gpu_ctx* c, int code, const std::string& m) {
  c->err = m;
  return code;
}
int cuda_fail(grains_gpu_ctx* c, cudaError_t e, const char* where) {
  c->err = std::string(where) + ": " + cudaGetErrorString(e);
  return GRAINS_GPU_CUDA_ERROR;
}
#define CK(call)                                                 \
  do {                                                           \
    cudaError_t e_ = (call);                                     \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call);       \
  } while (0)

// ---- shapes ------------------------------------------------------------------
// Tetrahedron (0, a, b, c) volume and second moments (F. Tonon, "Explicit exact
// formulas for the 3-D tetrahedron inertia tensor in terms of its vertex
// coordinates", J. Math. Stat. 1(1), 2004), as used for polyhedra by
// GrainsExec::computeVolumeInertiaContrib (Base/src/GrainsExec.cpp:748-800).
void tetra_contrib(D3 a, D3 b, D3 cc, double& vol, double I[3]) {
  double x[4] = {0, a.x, b.x, cc.x}, y[4] = {0, a.y, b.y, cc.y}, z[4] = {0, a.z, b.z, cc.z};
  double det = std::fabs((x[1] - x[0]) * (y[2] - y[0]) * (z[3] - z[0]) + (y[1] - y[0]) * (z[2] - z[0]) * (x[3] - x[0]) +
                         (z[1] - z[0]) * (x[2] - x[0]) * (y[3] - y[0]) - (z[1] - z[0]) * (y[2] - y[0]) * (x[3] - x[0]) -
                         (x[1] - x[0]) * (z[2] - z[0]) * (y[3] - y[0]) - (y[1] - y[0]) * (x[2] - x[0]) * (z[3] - z[0]));
  vol += det / 6.;
  auto sq = [](const double* u) {
    return u[0] * u[0] + u[0] * u[1] + u[1] * u[1] + u[0] * u[2] + u[1] * u[2] + u[2] * u[2] + u[0] * u[3] +
           u[1] * u[3] + u[2] * u[3] + u[3] * u[3];
  };
  I[0] += det * (sq(y) + sq(z)) / 60.;
  I[1] += det * (sq(x) + sq(z)) / 60.;
  I[2] += det * (sq(x) + sq(y)) / 60.;
}

// support of a shape in its local frame (for the local bounding box)
D3 shape_support(const ShapeHost& s, D3 v) {
  LocalBody<double> B{};
  B.type = s.type;
  B.nverts = (int)s.verts.size() / 3;
  B.verts = s.verts.data();
  B.radius = s.radius;
  B.cyl_r = s.radius;
  B.cyl_hh = s.half_height;
  B.ext = v3<double>(s.ext.x, s.ext.y, s.ext.z);
  V3<double> r = support_local(B, v3<double>(v.x, v.y, v.z));
  return d3(r.x, r.y, r.z);
}

int build_shape(int type, const double* p, int np, ShapeHost& s, std::string& err) {
  s.type = type;
  s.params.assign(p, p + np);
  if (type == GRAINS_GPU_SPHERE) {
    if (np < 1 || !(p[0] > 0)) return err = "sphere needs a positive radius", GRAINS_GPU_INVALID_ARGUMENT;
    s.radius = p[0];
    s.volume = 4.0 * kPi * std::pow(s.radius, 3.) / 3.0;                           // Sphere.cpp:152-155
    s.circ = s.radius;                                                              // Sphere.cpp:78-81
    double I = 8.0 * kPi * std::pow(s.radius, 5.) / 15.0;                           // Sphere.cpp:61-70
    s.inertia[0] = s.inertia[1] = s.inertia[2] = I;
  } else if (type == GRAINS_GPU_BOX) {
    if (np < 3) return err = "box needs LX, LY, LZ", GRAINS_GPU_INVALID_ARGUMENT;
    s.ext = d3(std::fabs(p[0]) / 2., std::fabs(p[1]) / 2., std::fabs(p[2]) / 2.);    // Box.cpp:27-33
    s.volume = 8.0 * s.ext.x * s.ext.y * s.ext.z;                                    // Box.cpp:286-292
    s.circ = xnorm(s.ext);                                                          // Box.cpp:230-233
    double e8 = 8.0 * s.ext.x * s.ext.y * s.ext.z;                                  // Box.cpp:181-210
    s.inertia[0] = e8 * (s.ext.y * s.ext.y + s.ext.z * s.ext.z) / 3.0;
    s.inertia[1] = e8 * (s.ext.x * s.ext.x + s.ext.z * s.ext.z) / 3.0;
    s.inertia[2] = e8 * (s.ext.y * s.ext.y + s.ext.x * s.ext.x) / 3.0;
  } else if (type == GRAINS_GPU_CYLINDER) {
    if (np < 2) return err = "cylinder needs radius and height", GRAINS_GPU_INVALID_ARGUMENT;
    s.radius = p[0];
    s.half_height = p[1] / 2.;
    s.volume = 2 * s.half_height * kPi * s.radius * s.radius;                       // Cylinder.cpp:97-100
    s.circ = std::sqrt(s.radius * s.radius + s.half_height * s.half_height);        // Cylinder.cpp:82-85
    double cst = 0.5 * s.half_height * s.radius * s.radius * kPi;                   // Cylinder.cpp:61-75
    s.inertia[0] = s.inertia[2] = cst * (4.0 * s.half_height * s.half_height / 3.0 + s.radius * s.radius);
    s.inertia[1] = 2.0 * cst * s.radius * s.radius;
  } else if (type == GRAINS_GPU_POLYHEDRON) {
    if (np < 1) return err = "polyhedron needs vertices", GRAINS_GPU_INVALID_ARGUMENT;
    int nv = (int)p[0], k = 1;
    if (nv < 4 || np < 1 + 3 * nv + 1) return err = "bad polyhedron description", GRAINS_GPU_INVALID_ARGUMENT;
    for (int i = 0; i < 3 * nv; ++i) s.verts.push_back(p[k++]);
    int nf = (int)p[k++];
    double I[3] = {0, 0, 0}, vol = 0;
    for (int f = 0; f < nf; ++f) {
      if (k >= np) return err = "truncated polyhedron faces", GRAINS_GPU_INVALID_ARGUMENT;
      int m = (int)p[k++];
      std::vector<int> face;
      for (int j = 0; j < m; ++j) {
        int vi = (int)p[k++];
        if (vi < 0 || vi >= nv) return err = "polyhedron face index out of range", GRAINS_GPU_INVALID_ARGUMENT;
        face.push_back(vi);
      }
      s.faces.push_back(face);
      auto V = [&](int i) { return d3(s.verts[3 * i], s.verts[3 * i + 1], s.verts[3 * i + 2]); };
      if (m == 3) {
        tetra_contrib(V(face[0]), V(face[1]), V(face[2]), vol, I);
      } else {  // fan around the face centroid (Polyhedron.cpp:341-356)
        D3 g = d3(0, 0, 0);
        for (int j = 0; j < m; ++j) g = d3(g.x + V(face[j]).x, g.y + V(face[j]).y, g.z + V(face[j]).z);
        g = d3(g.x / m, g.y / m, g.z / m);
        for (int j = 0, kk = m - 1; j < m; kk = j++) tetra_contrib(g, V(face[kk]), V(face[j]), vol, I);
      }
    }
    s.volume = vol;
    for (int i = 0; i < 3; ++i) s.inertia[i] = I[i];
    {
      std::vector<std::vector<int>> nb(nv);
      for (const auto& f : s.faces)
        for (size_t j = 0, kk = f.size() - 1; j < f.size(); kk = j++) nb[f[kk]].push_back(f[j]);
      s.adj_start.assign(1, 0);
      s.adj.clear();
      for (int i = 0; i < nv; ++i) {
        s.adj.insert(s.adj.end(), nb[i].begin(), nb[i].end());
        s.adj_start.push_back((int)s.adj.size());
      }
    }
    double r2 = 0;  // Polyhedron::computeCircumscribedRadius, Polyhedron.cpp:201-210
    for (int i = 0; i < nv; ++i) {
      double d = s.verts[3 * i] * s.verts[3 * i] + s.verts[3 * i + 1] * s.verts[3 * i + 1] +
                 s.verts[3 * i + 2] * s.verts[3 * i + 2];
      if (i == 0 || d > r2) r2 = d;
    }
    s.circ = std::sqrt(r2);
  } else {
    return err = "unknown shape type", GRAINS_GPU_INVALID_ARGUMENT;
  }
  // local bounding box half extents, Convex::bbox with the identity (Convex.cpp:29-41)
  for (int i = 0; i < 3; ++i) {
    D3 e = d3(i == 0, i == 1, i == 2);
    D3 ne = d3(-e.x, -e.y, -e.z);
    double mn = xdot(e, shape_support(s, ne)), mx = xdot(e, shape_support(s, e));
    s.lext[i] = (mx - mn) / 2.;
  }
  return 0;
}

ShapeDev shape_dev(const ShapeHost& s, int vert_offset) {
  ShapeDev d{};
  d.type = s.type;
  d.nverts = (int)s.verts.size() / 3;
  d.vert_offset = vert_offset;
  d.radius = s.radius;
  d.half_height = s.half_height;
  d.ext[0] = s.ext.x;
  d.ext[1] = s.ext.y;
  d.ext[2] = s.ext.z;
  d.circ = s.circ;
  for (int i = 0; i < 3; ++i) d.scaling_ext[i] = s.lext[i];
  d.volume = s.volume;
  return d;
}

// ---- obstacles ----------------------------------------------------------------
// ObstacleImposedVelocity's XML constructor (ObstacleImposedVelocity.cpp:60-262):
// directions normalised (Vector3::normalize), phases to radians, multi-sin
// amplitudes times the direction
LoadingDev loading_dev(const grains_gpu_obstacle_loading& g) {
  LoadingDev L{};
  L.type = g.type;
  L.has_center = g.has_center ? 1 : 0;
  L.ts = g.t_start;
  L.te = g.t_end;
  for (int i = 0; i < 3; ++i) L.center[i] = g.center[i];
  if (g.type == GRAINS_GPU_CONSTANT_TRANSLATION)
    for (int i = 0; i < 3; ++i) L.vel[i] = g.vector[i];
  if (g.type == GRAINS_GPU_CONSTANT_ROTATION)
    for (int i = 0; i < 3; ++i) L.omega[i] = g.vector[i];
  if (g.type == GRAINS_GPU_FORCE_TRANSLATION) {  // ObstacleImposedForce.cpp:55-68
    const double nv = std::sqrt(g.vector[0] * g.vector[0] + g.vector[1] * g.vector[1] + g.vector[2] * g.vector[2]);
    for (int i = 0; i < 3; ++i) {
      L.vel[i] = g.vector[i];
      L.unit[i] = g.vector[i] / nv;
    }
    L.amp = g.amplitude[0] > 0. ? g.amplitude[0] : 0.;
    L.period = g.amplitude[1];
  }
  if (g.type == GRAINS_GPU_SIN_TRANSLATION || g.type == GRAINS_GPU_CRENEL_TRANSLATION ||
      g.type == GRAINS_GPU_MULTISIN_TRANSLATION) {
    const double nv = std::sqrt(g.vector[0] * g.vector[0] + g.vector[1] * g.vector[1] + g.vector[2] * g.vector[2]);
    for (int i = 0; i < 3; ++i) L.unit[i] = g.vector[i] / nv;
    L.amp = g.amplitude[0];
    L.period = g.period[0];
    L.phase = g.phase_deg[0] * kPi / 180.;
    for (int i = 0; i < 3; ++i) {
      L.mper[i] = g.period[i];
      L.mphase[i] = g.phase_deg[i] * kPi / 180.;
      L.mamp[i] = g.amplitude[i] * L.unit[i];
    }
  }
  return L;
}

// an obstacle's legacy motion fields as one loading over [0, 1e9]
grains_gpu_obstacle_loading legacy_loading(const grains_gpu_obstacle& o) {
  grains_gpu_obstacle_loading g{};
  g.obstacle_id = o.id;
  g.t_start = 0.;
  g.t_end = 1.e9;
  if (o.omega[0] != 0. || o.omega[1] != 0. || o.omega[2] != 0.) {
    g.type = GRAINS_GPU_CONSTANT_ROTATION;
    for (int i = 0; i < 3; ++i) {
      g.vector[i] = o.omega[i];
      g.center[i] = o.rotation_center[i];
    }
    g.has_center = 1;
  } else {
    g.type = GRAINS_GPU_CONSTANT_TRANSLATION;
    for (int i = 0; i < 3; ++i) g.vector[i] = o.velocity[i];
  }
  return g;
}

// the loadings of one obstacle in ObstacleKinematicsVelocity's order
// (ObstacleKinematicsVelocity.cpp:28-40): by start time, a later-given
// loading before those starting at the same time
std::vector<LoadingDev> obstacle_loadings(const SysHost& s, const grains_gpu_obstacle& o) {
  std::vector<grains_gpu_obstacle_loading> v;
  auto insert = [&](const grains_gpu_obstacle_loading& g) {
    size_t k = 0;
    while (k < v.size() && v[k].t_start < g.t_start) ++k;
    v.insert(v.begin() + (long)k, g);
  };
  bool explicit_loads = false;
  for (const auto& g : s.loads)
    if (g.obstacle_id == o.id) {
      explicit_loads = true;
      if (g.type != GRAINS_GPU_FORCE_TRANSLATION) insert(g);
    }
  if (!explicit_loads && o.moving) v.push_back(legacy_loading(o));
  // the imposed forces after the velocities, in the order given
  // (ObstacleKinematicsForce::append, ObstacleKinematicsForce.cpp:27-30)
  for (const auto& g : s.loads)
    if (g.obstacle_id == o.id && g.type == GRAINS_GPU_FORCE_TRANSLATION) v.push_back(g);
  std::vector<LoadingDev> out;
  for (const auto& g : v) out.push_back(loading_dev(g));
  return out;
}

ObstacleDev obstacle_dev(const grains_gpu_obstacle& o, const ShapeHost& sh) {
  ObstacleDev d{};
  for (int i = 0; i < 9; ++i) d.b[i] = o.transform[i];
  for (int i = 0; i < 3; ++i) d.o[i] = o.transform[9 + i];
  for (int i = 0; i < 3; ++i) {
    // velocities are zero until the first move (Grains.cpp:124 sets them at
    // the start time, when an imposed motion starting then is not active yet)
    d.vel[i] = 0.;
    d.omega[i] = 0.;
  }
  d.crust = o.crust;
  d.circ = sh.circ;
  for (int i = 0; i < 3; ++i) d.scaling[i] = sh.lext[i] < kEpsilon ? 1. : (sh.lext[i] - o.crust) / sh.lext[i];
  d.id = o.id;
  d.material = o.material;
  d.shape = o.shape;
  d.moving = 0;  // set with its loadings
  // world AABB: Convex::bbox (Convex.cpp:29-41) -> BBox centre / extent (BBox.cpp:235-239)
  M3 b;
  for (int i = 0; i < 9; ++i) b.m[i] = d.b[i];
  double mn[3], mx[3];
  for (int i = 0; i < 3; ++i) {
    D3 r = mrow(b, i);
    D3 nr = d3(-r.x, -r.y, -r.z);
    mn[i] = xadd(d.o[i], xdot(r, shape_support(sh, nr)));
    mx[i] = xadd(d.o[i], xdot(r, shape_support(sh, r)));
  }
  for (int i = 0; i < 3; ++i) {
    d.bbe[i] = xdiv(xsub(mx[i], mn[i]), 2.);
    d.bbc[i] = xadd(mn[i], d.bbe[i]);
  }
  return d;
}

BodyRef obstacle_body(const ObstacleDev& o, const ShapeHost& sh) {
  BodyRef b{};
  b.type = sh.type;
  b.nverts = (int)sh.verts.size() / 3;
  b.verts = sh.verts.data();
  b.radius = sh.circ;
  b.cyl_r = sh.radius;
  b.cyl_hh = sh.half_height;
  b.ext = sh.ext;
  b.crust = o.crust;
  for (int i = 0; i < 9; ++i) b.basis.m[i] = o.b[i];
  b.origin = d3(o.o[0], o.o[1], o.o[2]);
  for (int i = 0; i < 3; ++i) {
    b.scaling[i] = o.scaling[i];
    b.lext[i] = sh.lext[i];
  }
  if (sh.type == GRAINS_GPU_POLYHEDRON && !sh.adj_start.empty()) {
    b.adj_start = sh.adj_start.data();
    b.adj = sh.adj.data();
  }
  return b;
}

// LinkedCell::Link(Obstacle*) (Base/src/LinkedCell.cpp:1371-1445): a cell is
// linked to a static obstacle when the obstacle's AABB is within one cell edge
// of the cell centre and a crust GJK test between the twice-expanded cell box
// and the obstacle says contact (RigidBodyWithCrust::isContact,
// RigidBodyWithCrust.cpp:842-956: distance < crust_cell + crust_obs - EPSILON).
void link_static_obstacles(const SysHost& s, const std::vector<ShapeHost>& shapes,
                           const std::vector<ObstacleDev>& obs, int first_obs,
                           std::vector<std::vector<int>>& cell_lists, double tol, bool accel) {
  const double hx = 0.5 * 2. * s.ex, hy = 0.5 * 2. * s.ey, hz = 0.5 * 2. * s.ez;
  ShapeHost cellbox;
  std::string unused;
  const double cell_edges[3] = {2. * hx, 2. * hy, 2. * hz};
  build_shape(GRAINS_GPU_BOX, cell_edges, 3, cellbox, unused);
  const int nb = s.nbi * s.nbj * s.nbk;
  for (size_t oi = 0; oi < s.obs.size(); ++oi) {
    const ObstacleDev& O = obs[first_obs + oi];
    if (O.moving) continue;
    const ShapeHost& sh = shapes[O.shape];
    BodyRef B = obstacle_body(O, sh);
    for (int c = 0; c < nb; ++c) {
      int i = c % s.nbi, k = (c / s.nbi) % s.nbk, j = c / (s.nbi * s.nbk);
      D3 cg = d3(s.dom.origin[0] + i * s.ex + s.ex / 2., s.dom.origin[1] + j * s.ey + s.ey / 2.,
                 s.dom.origin[2] + k * s.ez + s.ez / 2.);  // Cell::setCentre, Cell.cpp:74-82
      if (!in_zone(d3(O.bbc[0], O.bbc[1], O.bbc[2]), d3(O.bbe[0], O.bbe[1], O.bbe[2]), cg, hx, hy, hz)) continue;
      bool add;
      if (sh.type == GRAINS_GPU_SPHERE) {
        add = true;
      } else {
        BodyRef A{};
        A.type = GRAINS_GPU_BOX;
        A.verts = nullptr;
        A.radius = cellbox.circ;
        A.ext = cellbox.ext;
        A.crust = O.crust;
        for (int t = 0; t < 9; ++t) A.basis.m[t] = (t % 4 == 0) ? 1. : 0.;
        A.origin = cg;
        for (int t = 0; t < 3; ++t) {
          A.lext[t] = cellbox.lext[t];
          A.scaling[t] = cellbox.lext[t] < kEpsilon ? 1. : (cellbox.lext[t] - A.crust) / cellbox.lext[t];
        }
        add = false;
        D3 g = xsub3(A.origin, B.origin);
        if (xnorm(g) < A.radius + B.radius) {
          LocalBody<double> la = local_body<double>(A, d3(0, 0, 0), A.scaling);
          LocalBody<double> lb = local_body<double>(B, d3(0, 0, 0), B.scaling);
          GjkStart<double> st;
          st.accel = accel;
          GjkResult<double> r = gjk_distance(la, lb, tol, st);
          add = r.dist < A.crust + B.crust - kEpsilon;
        }
      }
      if (add) cell_lists[c].push_back(first_obs + (int)oi);
    }
  }
}

template <typename R>
void fill_arrays(grains_gpu_ctx* c, ParticleArrays<R>& P, int which) {
  auto& b = c->buf[which];
  P.xr = b.xr;
  P.q = b.q;
  P.basis = b.basis;
  P.v = (typename Vec4<R>::type*)b.v;
  P.w = (typename Vec4<R>::type*)b.w;
  P.wbf = (typename Vec4<R>::type*)b.wbf;
  P.F = (typename Vec4<R>::type*)b.F;
  P.T = (typename Vec4<R>::type*)b.T;
  P.inertia = (typename Vec4<R>::type*)b.inertia;
  P.md = b.md;
  P.meta = b.meta;
  P.orig = b.orig;
  P.key = b.key;
}

template <typename R>
StepArgs<R> make_args(grains_gpu_ctx* c) {
  StepArgs<R> a{};
  a.n = (int)c->n;
  a.n_cells = c->n_cells;
  a.n_sys = (int)c->sys.size();
  a.hist_cap = c->hist_cap;
  a.has_basis = c->has_basis ? 1 : 0;
  a.has_convex = c->has_convex ? 1 : 0;
  a.sys = c->d_sys;
  a.shapes = c->d_shapes;
  a.verts = c->d_verts;
  a.adj_start = c->d_adj_start;
  a.adj = c->d_adj;
  a.obs = c->d_obs;
  a.cell_obs_start = c->d_cell_obs_start;
  a.cell_obs_idx = c->d_cell_obs_idx;
  a.moving_idx = c->d_moving;
  a.loads = c->d_loads;
  a.load_flags = c->d_load_flags;
  a.laws = (const LawParams<R>*)c->d_laws;
  fill_arrays<R>(c, a.cur, c->cur);
  fill_arrays<R>(c, a.alt, 1 - c->cur);
  a.coord = c->coord;
  a.cell_count = c->cell_count;
  a.cell_start = c->cell_start;
  a.cell_cursor = c->cell_cursor;
  a.block_sums = c->block_sums;
  a.perm = c->perm;
  a.hist_prev = (HistEntry<R>*)c->hist[c->hcur];
  a.hist_n_prev = c->hist_n[c->hcur];
  a.hist_next = (HistEntry<R>*)c->hist[1 - c->hcur];
  a.hist_n_next = c->hist_n[1 - c->hcur];
  a.stats = c->stats;
  a.clist = c->clist;
  a.ccount = c->ccount;
  a.clist_cap = c->clist_cap;
  a.res_f = (typename Vec4<R>::type*)c->res_f;
  a.res_t = (typename Vec4<R>::type*)c->res_t;
  a.work = c->work;
  a.work_n = c->work_n;
  // the signed-volume GJK keeps its runs in the pair kernel
  a.gjk_out = c->gjk_sv ? nullptr : c->gjk_out;
  a.gjk_next = c->gjk_next;
  a.gjk_order = c->gjk_order;
  a.gjk_bins = c->gjk_bins;
  a.pairs = c->pairs;
  a.pairs_cap = c->pairs_cap;
  a.pairs_n = c->pairs_n;
  a.pair_force = c->pair_force;
  a.pair_sys = c->pair_sys;
  a.gjk_tol = c->gjk_tol;
  a.fluid_corrected = c->fluid_corrected;
  a.hydro = c->hydro_on ? c->d_hydro : nullptr;
  a.gjk_sv = c->gjk_sv;
  a.gjk_accel = c->gjk_accel;
  a.gjk_history = c->gjk_history;
  a.gdir_prev = c->gdir[c->hcur];
  a.gdir_n_prev = c->gdir_n[c->hcur];
  a.gdir_next = c->gdir[1 - c->hcur];
  a.gdir_n_next = c->gdir_n[1 - c->hcur];
  a.barrier_polls = c->barrier_polls;
  a.barrier_skip_block = c->barrier_skip_block;
  a.contacts_block = c->contacts_block;
  a.forces_block = c->forces_block;
  return a;
}

// Runs f(args) with the StepArgs of the context's precision
template <typename F>
int with_args(grains_gpu_ctx* c, F f) {
  if (c->precision == GRAINS_GPU_FP64) {
    StepArgs<double> a = make_args<double>(c);
    return f(a);
  }
  StepArgs<float> a = make_args<float>(c);
  return f(a);
}

// Cell ranges and permutation of the current positions; with gather the
// particle arrays are also permuted into cell order (other buffer).
int sort_now(grains_gpu_ctx* c, int gather_forces, bool gather = true) {
  int rc = 0;
  if (!c->keys_valid) {
    CK(cudaMemsetAsync(c->cell_count, 0, (size_t)c->n_cells * sizeof(int), c->stream));
    rc = with_args(c, [&](auto& a) { return launch_bin(a, c->stream); });
    if (rc) return fail(c, rc, "bin kernel launch failed");
  }
  rc = with_args(c, [&](auto& a) { return launch_sort_and_gather(a, c->stream, gather ? 1 : 0, gather_forces); });
  if (rc) return fail(c, rc, "sort kernels launch failed");
  if (gather) {
    c->cur = 1 - c->cur;
    c->since_gather = 0;
  } else {
    ++c->since_gather;
  }
  c->sorted = true;
  c->keys_valid = false;
  return 0;
}

// the sort of a middle step: the arrays are gathered every gather_every steps
int sort_for_step(grains_gpu_ctx* c) { return sort_now(c, 0, c->since_gather + 1 >= c->gather_every); }

int read_status(grains_gpu_ctx* c) {
  int st = 0;
  CK(cudaMemcpyAsync(&st, &c->stats->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return st;
}

std::string status_message(int st) {
  std::string m;
  if (st & GRAINS_GPU_CONTACT_ERROR) m += "ContactError (overlap exceeded the crust sum); ";
  if (st & GRAINS_GPU_MOTION_ERROR) m += "MotionError (displacement larger than the crust); ";
  if (st & GRAINS_GPU_OUT_OF_GRID) m += "SimulationError (particle outside the linked-cell grid); ";
  if (st & GRAINS_GPU_HISTORY_FULL) m += "contact-memory row full; ";
  if (st & GRAINS_GPU_GJK_NOT_CONVERGED) m += "GJK iteration cap reached; ";
  return m;
}

// errors that end a run (informational bits excluded)
int fatal_bits(int st) { return st & ~(GRAINS_GPU_CONTACT_HANDLED | GRAINS_GPU_GJK_NOT_CONVERGED); }

int finish_call(grains_gpu_ctx* c) {
  int st = read_status(c);
  if (st < 0) return GRAINS_GPU_CUDA_ERROR;
  int f = fatal_bits(st);
  if (f) c->err = status_message(st);
  return f;
}

int flush_kick(grains_gpu_ctx* c) {
  if (!c->pending_kick2) return 0;
  int rc = with_args(c, [&](auto& a) { return launch_kick_move(a, c->stream, 1, c->pending_dt, 0, 0., 0.); });
  c->pending_kick2 = false;
  return rc ? fail(c, rc, "advance-velocity launch failed") : 0;
}

int forces_now(grains_gpu_ctx* c, double dt, int diag, int phases = 7, int kick = 0) {
  if (!c->sorted) {
    if (int rc = sort_now(c, 1)) return rc;
  }
  int rc = with_args(c, [&](auto& a) { return launch_forces(a, c->stream, dt, diag, phases, kick); });
  if (rc) return fail(c, rc, "force kernel launch failed");
  if (phases & 4) c->hcur = 1 - c->hcur;
  if (phases & 2) c->obs_force_valid = true;
  return 0;
}

// moving obstacles follow the particles' drift (AllComponents::Move,
// AllComponents.cpp:166-215)
// from_host: 'time' is the clock after this step's increment, given by the
// host (and stored in the device clock); otherwise the device clock advances
// by dt, as Grains::Simulation advances m_time
int move_obstacles(grains_gpu_ctx* c, double dt, int from_host = 0, double time = 0.) {
  if (c->n_moving == 0) return 0;
  if (c->n_force_obs > 0) {
    // the contact forces on the force-driven obstacles from the last force
    // evaluation (zero before the first one, like the reference's torsors)
    if (c->obs_force_valid) {
      int rc = with_args(c, [&](auto& a) {
        return launch_obstacle_force(a, c->d_force_part, (int)c->h_obs.size(), c->stream);
      });
      if (rc) return fail(c, rc, "obstacle force launch failed");
    } else {
      CK(cudaMemsetAsync(c->d_force_part, 0, (size_t)kForceBlocks * kMaxForceObstacles * 3 * sizeof(double),
                         c->stream));
    }
  }
  int rc = launch_obstacle_move(c->d_obs, c->d_moving, c->n_moving, c->d_loads, c->d_load_flags,
                                (int)c->sys.size(), c->d_shapes, c->d_verts, dt, c->clock, time, from_host,
                                c->d_force_part, c->d_force_pid, c->stream);
  return rc ? fail(c, rc, "obstacle move launch failed") : 0;
}

// First step of a run: move (finishing a pending second half kick), keys
int first_move(grains_gpu_ctx* c, double dt, double time) {
  int rc = with_args(c, [&](auto& a) {
    return launch_kick_move(a, c->stream, c->pending_kick2 ? 1 : 0, c->pending_dt, 1, 0.5 * dt, dt);
  });
  if (rc) return fail(c, rc, "kick/move launch failed");
  c->pending_kick2 = false;
  c->keys_valid = true;
  c->sorted = false;
  return move_obstacles(c, dt, 1, time + dt);
}

// A middle step: sort, contact lists, contact law, then the per-particle sums
// with the rest of the step (second half kick) and the next step's first half
// kick, drift and binning in the same kernel.  (Folding that kick into the
// contact-law kernel of an earlier design, one thread per particle evaluating
// every contact, was 14-15 % slower per step on 200,000 spheres; the sums
// kernel is light, and the fold saves the torsor's round trip and a launch.)
int middle_step(grains_gpu_ctx* c, double dt) {
  if (int rc = sort_for_step(c)) return rc;
  if (int rc = forces_now(c, dt, 0, 7, 1)) return rc;
  c->keys_valid = true;
  c->sorted = false;
  return move_obstacles(c, dt);
}

// n middle steps in one cooperative launch (persistent_steps_kernel); the
// host then follows the buffer selection the launch leaves
int persistent_middle_steps(grains_gpu_ctx* c, int n, double dt) {
  if (!c->pbar) {
    void* q = nullptr;
    CK(cudaMalloc(&q, 2 * sizeof(unsigned)));
    c->pbar = (unsigned*)q;
  }
  if (!c->pblocks) {
    c->pblocks = with_args(c, [&](auto& a) { return persistent_blocks(a); });
    if (c->pblocks <= 0) return fail(c, GRAINS_GPU_CUDA_ERROR, "persistent launch: occupancy query failed");
    void* q = nullptr;
    CK(cudaMalloc(&q, (size_t)c->pblocks * sizeof(int)));
    c->psums = (int*)q;
  }
  CK(cudaMemsetAsync(c->pbar, 0, 2 * sizeof(unsigned), c->stream));
  int rc = with_args(c, [&](auto& a) {
    return launch_persistent_steps(a, c->stream, n, dt, c->gather_every, c->since_gather, c->n_moving, c->clock,
                                   c->pbar, c->psums, c->pblocks);
  });
  if (rc) return fail(c, rc, "persistent launch failed (cooperative launch refused?)");
  for (int k = 0; k < n; ++k) {
    if (c->since_gather + 1 >= c->gather_every) {
      c->cur = 1 - c->cur;
      c->since_gather = 0;
    } else {
      ++c->since_gather;
    }
    c->hcur = 1 - c->hcur;
  }
  c->keys_valid = true;
  c->sorted = false;
  return 0;
}

// The last step of a run: sort and forces; the second half kick stays pending
int last_step(grains_gpu_ctx* c, double dt) {
  if (int rc = sort_now(c, 0)) return rc;
  if (int rc = forces_now(c, dt, 0)) return rc;
  c->pending_kick2 = true;
  c->pending_dt = 0.5 * dt;
  return 0;
}

// Contact-list scratch for cap_per entries per particle: the lists, the
// result of each entry (two R4) and the work items; grown, never shrunk.
int ensure_lists(grains_gpu_ctx* c, int cap_per) {
  const int64_t need = (int64_t)c->cap * cap_per;
  if (need > c->clist_alloc || (c->has_convex && !c->gjk_out)) {
    for (void** p : {(void**)&c->clist, &c->res_f, &c->res_t, (void**)&c->work, (void**)&c->gjk_out,
                     (void**)&c->gjk_order})
      if (*p) {
        cudaFree(*p);
        *p = nullptr;
      }
    c->clist_alloc = 0;
    c->obs_force_valid = false;  // the new lists hold no force evaluation yet
    const size_t r4 = 4 * c->rsize;
    void* q = nullptr;
    CK(cudaMalloc(&q, (size_t)need * sizeof(int)));
    c->clist = (int*)q;
    CK(cudaMalloc(&q, (size_t)need * r4));
    c->res_f = q;
    CK(cudaMalloc(&q, (size_t)need * r4));
    c->res_t = q;
    CK(cudaMalloc(&q, (size_t)need * sizeof(int4)));
    c->work = (int4*)q;
    if (c->has_convex) {  // one narrowphase result per possible work item, their order
      CK(cudaMalloc(&q, (size_t)need * sizeof(GjkOut)));
      c->gjk_out = (GjkOut*)q;
      CK(cudaMalloc(&q, (size_t)need * sizeof(int)));
      c->gjk_order = (int*)q;
    }
    c->clist_alloc = need;
    for (int k = 0; k < 4; ++k)  // graphs hold the old pointers
      if (c->graph[k]) {
        cudaGraphExecDestroy(c->graph[k]);
        c->graph[k] = nullptr;
      }
  }
  c->clist_cap = cap_per;
  return 0;
}

// LinkedCell::set (LinkedCell.cpp:69-98) with the cell edge scaled by the
// context's cell factor (1 = the reference's grid)
int apply_grid(grains_gpu_ctx* c, SysHost& s) {
  const grains_gpu_domain* d = &s.dom;
  const double cs = d->cell_size * c->cell_factor;
  if (cs > kEpsilon) {
    s.nbi = (int)((d->size[0] + kEpsilon) / cs);
    if (!s.nbi) s.nbi = 1;
    s.ex = d->size[0] / s.nbi;
    s.nbj = (int)((d->size[1] + kEpsilon) / cs);
    if (!s.nbj) s.nbj = 1;
    s.ey = d->size[1] / s.nbj;
    s.nbk = (int)((d->size[2] + kEpsilon) / cs);
    if (!s.nbk) s.nbk = 1;
    s.ez = d->size[2] / s.nbk;
  } else {
    s.nbi = s.nbj = s.nbk = 1;
    s.ex = d->size[0];
    s.ey = d->size[1];
    s.ez = d->size[2];
  }
  if ((double)s.nbi * s.nbj * s.nbk > 2.0e9) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "too many cells");
  return 0;
}
}  // namespace

// ===========================================================================
extern "C" {

int grains_gpu_create(const grains_gpu_config* cfg, grains_gpu_ctx** out) {
  if (!cfg || !out) return GRAINS_GPU_INVALID_ARGUMENT;
  *out = nullptr;
  if (cfg->n_systems < 1 || cfg->max_particles < 1 || cfg->max_particles > (int64_t)1 << 30)
    return GRAINS_GPU_INVALID_ARGUMENT;
  if (cfg->precision != GRAINS_GPU_FP64 && cfg->precision != GRAINS_GPU_MIXED) return GRAINS_GPU_INVALID_ARGUMENT;
  grains_gpu_ctx* c = new grains_gpu_ctx();
  c->cfg = *cfg;
  c->precision = cfg->precision;
  c->hist_cap = cfg->history_capacity > 0 ? cfg->history_capacity : 24;
  c->rsize = cfg->precision == GRAINS_GPU_FP64 ? 8 : 4;
  c->cap = cfg->max_particles;
  c->sys.resize(cfg->n_systems);
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    int rc = cuda_fail(c, e, "cudaSetDevice/cudaStreamCreate");
    *out = c;  // keep the message readable
    return rc;
  }
  const size_t N = (size_t)c->cap;
  const size_t r4 = 4 * c->rsize;
  bool ok = true;
  for (int k = 0; k < 2 && ok; ++k) {
    auto& b = c->buf[k];
    b.xr = dalloc<double4>(N, c->pool);
    b.q = dalloc<double4>(N, c->pool);
    b.basis = nullptr;
    b.v = dalloc<char>(N * r4, c->pool);
    b.w = dalloc<char>(N * r4, c->pool);
    b.wbf = dalloc<char>(N * r4, c->pool);
    b.F = dalloc<char>(N * r4, c->pool);
    b.T = dalloc<char>(N * r4, c->pool);
    b.inertia = dalloc<char>(N * r4, c->pool);
    b.md = dalloc<double4>(N, c->pool);
    b.meta = dalloc<int4>(N, c->pool);
    b.orig = dalloc<int>(N, c->pool);
    b.key = dalloc<unsigned>(N, c->pool);
    ok = b.xr && b.q && b.v && b.w && b.wbf && b.F && b.T && b.inertia && b.md && b.meta && b.orig && b.key;
  }
  const size_t hsz = c->precision == GRAINS_GPU_FP64 ? sizeof(HistEntry<double>) : sizeof(HistEntry<float>);
  for (int k = 0; k < 2 && ok; ++k) {
    c->hist[k] = dalloc<char>(N * c->hist_cap * hsz, c->pool);
    c->hist_n[k] = dalloc<int>(N, c->pool);
    ok = c->hist[k] && c->hist_n[k];
  }
  if (ok) {
    c->coord = dalloc<int>(N, c->pool);
    c->perm = dalloc<int>(N, c->pool);
    c->stats = dalloc<StatsDev>(1, c->pool);
    c->pairs_cap = (int)std::min<size_t>(16 * N + 1024, (size_t)1 << 30);
    c->pairs = dalloc<int>(2 * (size_t)c->pairs_cap, c->pool);
    c->pairs_n = dalloc<unsigned long long>(1, c->pool);
    c->pair_force = dalloc<double>(3 * (size_t)c->pairs_cap, c->pool);
    c->pair_sys = dalloc<int>((size_t)c->pairs_cap, c->pool);
    c->clock = dalloc<double>(1, c->pool);
    c->work_n = dalloc<int>(1, c->pool);
    c->gjk_next = dalloc<int>(1, c->pool);
    c->gjk_bins = dalloc<int>(64, c->pool);
    ok = c->coord && c->perm && c->stats && c->pairs && c->pairs_n && c->pair_force && c->pair_sys && c->clock &&
         c->work_n && c->gjk_next && c->gjk_bins;
  }
  if (!ok) {
    c->err = "cudaMalloc failed for the requested capacity";
    *out = c;
    return GRAINS_GPU_CUDA_ERROR;
  }
  for (int k = 0; k < 2; ++k) cudaMemsetAsync(c->hist_n[k], 0, N * sizeof(int), c->stream);
  cudaMemsetAsync(c->perm, 0, N * sizeof(int), c->stream);
  cudaMemsetAsync(c->stats, 0, sizeof(StatsDev), c->stream);
  cudaMemsetAsync(c->work_n, 0, sizeof(int), c->stream);
  cudaMemsetAsync(c->gjk_next, 0, sizeof(int), c->stream);
  cudaStreamSynchronize(c->stream);
  *out = c;
  return 0;
}

int grains_gpu_destroy(grains_gpu_ctx* c) {
  if (!c) return 0;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int k = 0; k < 4; ++k)
    if (c->graph[k]) cudaGraphExecDestroy(c->graph[k]);
  for (void* p : c->pool) cudaFree(p);
  for (void* p : c->table_pool) cudaFree(p);
  for (int k = 0; k < 2; ++k)
    if (c->buf[k].basis) cudaFree(c->buf[k].basis);
  if (c->stage) cudaFree(c->stage);
  if (c->row_scratch) cudaFree(c->row_scratch);
  if (c->d_hydro) cudaFree(c->d_hydro);
  for (void* p : {(void*)c->clist, (void*)c->ccount, c->res_f, c->res_t, (void*)c->work, (void*)c->gjk_out,
                  (void*)c->gjk_order})
    if (p) cudaFree(p);
  if (c->pbar) cudaFree(c->pbar);
  if (c->psums) cudaFree(c->psums);
  for (void* p : {(void*)c->d_row_id, (void*)c->d_row_sys, (void*)c->d_row_keys, (void*)c->d_key_rows,
                  (void*)c->d_attr})
    if (p) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int grains_gpu_last_error(const grains_gpu_ctx* c, char* buf, size_t len) {
  if (!c || !buf || !len) return GRAINS_GPU_INVALID_ARGUMENT;
  std::snprintf(buf, len, "%s", c->err.c_str());
  return 0;
}

int grains_gpu_get_stream(const grains_gpu_ctx* c, void** stream) {
  if (!c || !stream) return GRAINS_GPU_INVALID_ARGUMENT;
  *stream = (void*)c->stream;
  return 0;
}

int grains_gpu_set_domain(grains_gpu_ctx* c, int32_t system, const grains_gpu_domain* d) {
  if (!c || !d) return GRAINS_GPU_INVALID_ARGUMENT;
  if (system < 0 || system >= (int)c->sys.size()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "bad system index");
  for (int i = 0; i < 3; ++i)
    if (!(d->size[i] > 0)) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "domain size must be positive");
  SysHost& s = c->sys[system];
  s.dom = *d;
  if (int rc = apply_grid(c, s)) return rc;
  s.has_domain = true;
  c->uploaded = false;
  c->tables_dirty = true;
  return 0;
}

int grains_gpu_add_shape(grains_gpu_ctx* c, int32_t type, const double* params, int32_t n, int32_t* id) {
  if (!c || !params || !id) return GRAINS_GPU_INVALID_ARGUMENT;
  ShapeHost s;
  std::string err;
  if (int rc = build_shape(type, params, n, s, err)) return fail(c, rc, err);
  c->shapes.push_back(s);
  *id = (int32_t)c->shapes.size() - 1;
  c->tables_dirty = true;
  return 0;
}

int grains_gpu_set_contact_law(grains_gpu_ctx* c, int32_t system, int32_t a, int32_t b, int32_t law,
                               const double* p, int32_t n) {
  if (!c || !p) return GRAINS_GPU_INVALID_ARGUMENT;
  if (system < 0 || system >= (int)c->sys.size() || a < 0 || b < 0)
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "bad system or material index");
  int maxmat = c->cfg.max_materials > 0 ? c->cfg.max_materials : 4;
  if (a >= maxmat || b >= maxmat) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "material index >= max_materials");
  LawHost L;
  L.type = law;
  if (law == GRAINS_GPU_HOOKE_MEMORY) {
    if (n < 8) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "HookeMemory needs kn, en, etat, muc, kt, mur, etarpf, epst");
    for (int i = 0; i < 8; ++i) L.p[i] = p[i];
  } else if (law == GRAINS_GPU_HOOKE) {
    if (n < 5) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "Hooke needs kn, en, etat, muc, kr");
    L.p[0] = p[0];
    L.p[1] = p[1];
    L.p[2] = p[2];
    L.p[3] = p[3];
    L.p[8] = p[4];
  } else if (law == GRAINS_GPU_HERTZ) {
    // HertzContactForceModel::defineParameters (HertzContactForceModel.cpp:236-276)
    if (n < 5) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "Hertz needs Es, en, muc, kr, Gs");
    L.p[9] = p[0];
    L.p[1] = p[1];
    L.p[3] = p[2];
    L.p[8] = p[3];
    L.p[10] = p[4];
  } else if (law == GRAINS_GPU_HERTZ_MEMORY) {
    // HertzMemoryContactForceModel::defineParameters (HertzMemoryContactForceModel.cpp:261-309)
    if (n < 7) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "HertzMemory needs Es, en, muc, Gs, mur, etarpf, epst");
    L.p[9] = p[0];
    L.p[1] = p[1];
    L.p[3] = p[2];
    L.p[10] = p[3];
    L.p[5] = p[4];
    L.p[6] = p[5];
    L.p[7] = p[6];
  } else {
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "unknown contact law");
  }
  if ((law == GRAINS_GPU_HERTZ || law == GRAINS_GPU_HERTZ_MEMORY) && !(L.p[9] > 0 && L.p[10] > 0))
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "Hertz laws need Es > 0 and Gs > 0");
  if (!(L.p[1] > 0 && L.p[1] <= 1)) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "restitution must be in (0, 1]");
  // m_beta, HookeMemoryContactForceModel.cpp:28 / HookeContactForceModel.cpp:17
  L.beta = std::log(L.p[1]) / std::sqrt(kPi * kPi + std::log(L.p[1]) * std::log(L.p[1]));
  c->sys[system].laws[std::make_pair(std::min(a, b), std::max(a, b))] = L;
  c->uploaded = false;
  c->tables_dirty = true;
  return 0;
}

int grains_gpu_set_obstacles(grains_gpu_ctx* c, int32_t system, int32_t n, const grains_gpu_obstacle* o) {
  if (!c || (n > 0 && !o)) return GRAINS_GPU_INVALID_ARGUMENT;
  if (system < 0 || system >= (int)c->sys.size()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "bad system index");
  const int maxmat = c->cfg.max_materials > 0 ? c->cfg.max_materials : 4;
  for (int i = 0; i < n; ++i) {
    if (o[i].shape < 0 || o[i].shape >= (int)c->shapes.size())
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "obstacle shape id out of range");
    if (o[i].material < 0 || o[i].material >= maxmat)
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "obstacle material out of range");
  }
  c->sys[system].obs.assign(o, o + n);
  c->uploaded = false;
  c->tables_dirty = true;
  return 0;
}

namespace {
void drop_graphs(grains_gpu_ctx* c) {
  for (int k = 0; k < 4; ++k)
    if (c->graph[k]) {
      cudaGraphExecDestroy(c->graph[k]);
      c->graph[k] = nullptr;
    }
}
}  // namespace

int grains_gpu_set_collision_algorithm(grains_gpu_ctx* c, int32_t algorithm) {
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  if (algorithm != GRAINS_GPU_GJK && algorithm != GRAINS_GPU_GJK_SV)
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "unknown collision algorithm");
  c->gjk_sv = algorithm == GRAINS_GPU_GJK_SV ? 1 : 0;
  drop_graphs(c);
  return 0;
}

int grains_gpu_set_collision_options(grains_gpu_ctx* c, double tolerance, int32_t acceleration, int32_t history) {
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!(tolerance >= 1e-10))  // Grains.cpp:684-689 rejects tolerances below 1e-10
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "GJK tolerance must be at least 1e-10");
  if ((acceleration != 0 && acceleration != 1) || (history != 0 && history != 1))
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "acceleration and history are 0 (OFF) or 1 (ON)");
  if (history && !c->gdir[0]) {
    const size_t N = (size_t)c->cap;
    for (int k = 0; k < 2; ++k) {
      c->gdir[k] = dalloc<GjkDir>(N * c->hist_cap, c->pool);
      c->gdir_n[k] = dalloc<int>(N, c->pool);
      if (!c->gdir[k] || !c->gdir_n[k]) return fail(c, GRAINS_GPU_CUDA_ERROR, "collision history allocation failed");
    }
  }
  if (history && !c->gjk_history)  // a history starts empty
    for (int k = 0; k < 2; ++k) CK(cudaMemsetAsync(c->gdir_n[k], 0, (size_t)c->cap * sizeof(int), c->stream));
  c->gjk_tol = tolerance;
  c->gjk_accel = acceleration;
  c->gjk_history = history;
  c->tables_dirty = true;  // the static obstacle-cell links use the same GJK
  drop_graphs(c);
  return 0;
}

int grains_gpu_set_obstacle_loadings(grains_gpu_ctx* c, int32_t system, int32_t n,
                                     const grains_gpu_obstacle_loading* l) {
  if (!c || n < 0 || (n && !l)) return GRAINS_GPU_INVALID_ARGUMENT;
  if (system < 0 || system >= (int)c->sys.size()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "bad system index");
  SysHost& s = c->sys[system];
  for (int k = 0; k < n; ++k) {
    bool found = false;
    for (const auto& o : s.obs) found = found || o.id == l[k].obstacle_id;
    if (!found) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "loading of an unknown obstacle");
    if (l[k].type < GRAINS_GPU_CONSTANT_TRANSLATION || l[k].type > GRAINS_GPU_FORCE_TRANSLATION)
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "unknown loading type");
    if (l[k].type == GRAINS_GPU_FORCE_TRANSLATION &&
        !(l[k].vector[0] != 0. || l[k].vector[1] != 0. || l[k].vector[2] != 0.))
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "an imposed force needs a non-zero force");
    if ((l[k].type == GRAINS_GPU_SIN_TRANSLATION || l[k].type == GRAINS_GPU_CRENEL_TRANSLATION) &&
        !(l[k].period[0] > 0.))
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "a periodic loading needs a positive period");
    if (l[k].type == GRAINS_GPU_MULTISIN_TRANSLATION &&
        !(l[k].period[0] > 0. && l[k].period[1] > 0. && l[k].period[2] > 0.))
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "a periodic loading needs a positive period");
  }
  s.loads.assign(l, l + n);
  c->uploaded = false;
  c->tables_dirty = true;
  return 0;
}

namespace {
// Builds the device tables and the per-cell obstacle links (set-up time)
int build_tables(grains_gpu_ctx* c) {
  for (void* p : c->table_pool) cudaFree(p);
  c->table_pool.clear();
  const int maxmat = c->cfg.max_materials > 0 ? c->cfg.max_materials : 4;
  std::vector<SysDev> hs;
  std::vector<ObstacleDev> ho;
  std::vector<LoadingDev> hl;
  std::vector<int> moving;
  int n_force = 0;  // force-driven obstacles
  std::vector<int> cstart;
  std::vector<int> cidx;
  int cells = 0;
  for (size_t si = 0; si < c->sys.size(); ++si) {
    SysHost& s = c->sys[si];
    if (!s.has_domain) return fail(c, GRAINS_GPU_NOT_READY, "a system has no domain");
    SysDev d{};
    d.ox = s.dom.origin[0];
    d.oy = s.dom.origin[1];
    d.oz = s.dom.origin[2];
    d.ex = s.ex;
    d.ey = s.ey;
    d.ez = s.ez;
    d.gx = s.dom.gravity[0];
    d.gy = s.dom.gravity[1];
    d.gz = s.dom.gravity[2];
    d.nbi = s.nbi;
    d.nbj = s.nbj;
    d.nbk = s.nbk;
    d.cell_offset = cells;
    d.law_offset = (int)si * maxmat * maxmat;
    d.n_mat = maxmat;
    d.obs_offset = (int)ho.size();
    d.n_obs = (int)s.obs.size();
    d.moving_offset = (int)moving.size();
    for (size_t k = 0; k < s.obs.size(); ++k) {
      ObstacleDev od = obstacle_dev(s.obs[k], c->shapes[s.obs[k].shape]);
      const std::vector<LoadingDev> ls = obstacle_loadings(s, s.obs[k]);
      od.load_first = (int)hl.size();
      od.load_count = (int)ls.size();
      od.moving = ls.empty() ? 0 : 1;
      od.sys = (int)si;
      od.force_slot = -1;
      od.moved = 0;
      for (const auto& L : ls)
        if (L.type == GRAINS_GPU_FORCE_TRANSLATION) od.force_slot = n_force;
      if (od.force_slot >= 0 && ++n_force > kMaxForceObstacles)
        return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "more force-driven obstacles than kMaxForceObstacles (4)");
      hl.insert(hl.end(), ls.begin(), ls.end());
      ho.push_back(od);
      if (od.moving) moving.push_back(d.obs_offset + (int)k);
    }
    d.n_moving = (int)moving.size() - d.moving_offset;
    const int nb = s.nbi * s.nbj * s.nbk;
    std::vector<std::vector<int>> lists(nb);
    link_static_obstacles(s, c->shapes, ho, d.obs_offset, lists, c->gjk_tol, c->gjk_accel != 0);
    for (int k = 0; k < nb; ++k) {
      cstart.push_back((int)cidx.size());
      cidx.insert(cidx.end(), lists[k].begin(), lists[k].end());
    }
    if ((long long)cells + nb > 2000000000LL) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "too many cells");
    cells += nb;
    hs.push_back(d);
  }
  cstart.push_back((int)cidx.size());
  c->n_cells = cells;
  c->n_moving = (int)moving.size();
  c->h_sys = hs;
  c->h_obs = ho;
  // laws
  std::vector<LawParams<double>> ld(c->sys.size() * maxmat * maxmat);
  std::vector<LawParams<float>> lf(ld.size());
  for (auto& x : ld) x.type = -1;
  for (auto& x : lf) x.type = -1;
  for (size_t si = 0; si < c->sys.size(); ++si)
    for (auto& kv : c->sys[si].laws)
      for (int flip = 0; flip < 2; ++flip) {
        int a = flip ? kv.first.second : kv.first.first, b = flip ? kv.first.first : kv.first.second;
        size_t k = si * maxmat * maxmat + a * maxmat + b;
        const LawHost& L = kv.second;
        LawParams<double> P{};
        P.type = L.type;
        P.kn = L.p[0];
        P.en = L.p[1];
        P.etat = L.p[2];
        P.muc = L.p[3];
        P.kt = L.p[4];
        P.mur = L.p[5];
        P.etarpf = L.p[6];
        P.epst = L.p[7];
        P.kr = L.p[8];
        P.Es = L.p[9];
        P.Gs = L.p[10];
        P.beta = L.beta;
        P.rolling = (law_has_memory(L.type) && P.mur != 0.) ? 1 : 0;
        P.kn64 = P.kn;
        P.beta64 = P.beta;
        P.etat64 = P.etat;
        P.Es64 = P.Es;
        P.Gs64 = P.Gs;
        ld[k] = P;
        LawParams<float> Q{};
        Q.type = P.type;
        Q.rolling = P.rolling;
        Q.kn = (float)P.kn; Q.en = (float)P.en; Q.etat = (float)P.etat; Q.muc = (float)P.muc;
        Q.kt = (float)P.kt; Q.mur = (float)P.mur; Q.etarpf = (float)P.etarpf; Q.epst = (float)P.epst;
        Q.kr = (float)P.kr; Q.beta = (float)P.beta;
        Q.Es = (float)P.Es; Q.Gs = (float)P.Gs;
        Q.kn64 = P.kn64; Q.beta64 = P.beta64; Q.etat64 = P.etat64; Q.Es64 = P.Es64; Q.Gs64 = P.Gs64;
        lf[k] = Q;
      }
  // shapes
  std::vector<ShapeDev> sd;
  std::vector<double> verts;
  std::vector<int> adj_start, adj;  // adjacency over the whole vertex table
  for (auto& s : c->shapes) {
    sd.push_back(shape_dev(s, (int)verts.size() / 3));
    verts.insert(verts.end(), s.verts.begin(), s.verts.end());
    const int nv = (int)s.verts.size() / 3;
    for (int i = 0; i < nv; ++i) {
      adj_start.push_back((int)adj.size());
      if (!s.adj_start.empty())
        adj.insert(adj.end(), s.adj.begin() + s.adj_start[i], s.adj.begin() + s.adj_start[i + 1]);
    }
  }
  adj_start.push_back((int)adj.size());
  auto up = [&](const void* src, size_t bytes, void** dst) -> int {
    void* p = nullptr;
    CK(cudaMalloc(&p, bytes ? bytes : 16));
    c->table_pool.push_back(p);
    if (bytes) CK(cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, c->stream));
    *dst = p;
    return 0;
  };
  int rc = 0;
  rc |= up(hs.data(), hs.size() * sizeof(SysDev), (void**)&c->d_sys);
  rc |= up(sd.data(), sd.size() * sizeof(ShapeDev), (void**)&c->d_shapes);
  rc |= up(verts.data(), verts.size() * sizeof(double), (void**)&c->d_verts);
  rc |= up(adj_start.data(), adj_start.size() * sizeof(int), (void**)&c->d_adj_start);
  rc |= up(adj.data(), adj.size() * sizeof(int), (void**)&c->d_adj);
  rc |= up(ho.data(), ho.size() * sizeof(ObstacleDev), (void**)&c->d_obs);
  rc |= up(cstart.data(), cstart.size() * sizeof(int), (void**)&c->d_cell_obs_start);
  rc |= up(cidx.data(), cidx.size() * sizeof(int), (void**)&c->d_cell_obs_idx);
  rc |= up(moving.data(), moving.size() * sizeof(int), (void**)&c->d_moving);
  rc |= up(hl.data(), hl.size() * sizeof(LoadingDev), (void**)&c->d_loads);
  {
    std::vector<int> flags(2 * c->sys.size(), 0);  // no loading active before the first step
    rc |= up(flags.data(), flags.size() * sizeof(int), (void**)&c->d_load_flags);
  }
  c->n_force_obs = n_force;
  c->d_force_part = c->d_force_pid = nullptr;
  if (n_force > 0) {
    std::vector<double> part((size_t)kForceBlocks * kMaxForceObstacles * 3, 0.);
    std::vector<double> pid(c->sys.size() * kForcePidWords, 0.);  // the controllers start without history
    rc |= up(part.data(), part.size() * sizeof(double), (void**)&c->d_force_part);
    rc |= up(pid.data(), pid.size() * sizeof(double), (void**)&c->d_force_pid);
  }
  {
    // obstacle ids by global obstacle index, and each system's first index
    std::vector<int> oid, ooff;
    for (const auto& sy : c->sys) {
      ooff.push_back((int)oid.size());
      for (const auto& o : sy.obs) oid.push_back(o.id);
    }
    rc |= up(oid.data(), oid.size() * sizeof(int), (void**)&c->d_obs_id);
    rc |= up(ooff.data(), ooff.size() * sizeof(int), (void**)&c->d_sys_obs_offset);
  }
  if (c->precision == GRAINS_GPU_FP64)
    rc |= up(ld.data(), ld.size() * sizeof(LawParams<double>), &c->d_laws);
  else
    rc |= up(lf.data(), lf.size() * sizeof(LawParams<float>), &c->d_laws);
  if (rc) return rc;
  // cell arrays
  void* p = nullptr;
  CK(cudaMalloc(&p, (size_t)cells * sizeof(int)));
  c->table_pool.push_back(p);
  c->cell_count = (int*)p;
  CK(cudaMalloc(&p, ((size_t)cells + 1) * sizeof(int)));
  c->table_pool.push_back(p);
  c->cell_start = (int*)p;
  CK(cudaMalloc(&p, ((size_t)cells + 1) * sizeof(int)));
  c->table_pool.push_back(p);
  c->cell_cursor = (int*)p;
  CK(cudaMalloc(&p, ((size_t)cells / 4096 + 2) * sizeof(int)));
  c->table_pool.push_back(p);
  c->block_sums = (int*)p;
  CK(cudaMemsetAsync(c->cell_count, 0, (size_t)cells * sizeof(int), c->stream));
  if (((size_t)cells / 4096 + 1) > 4096) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "too many cells for the scan");
  for (int k = 0; k < 4; ++k)
    if (c->graph[k]) {
      cudaGraphExecDestroy(c->graph[k]);
      c->graph[k] = nullptr;
    }
  return 0;
}
}  // namespace

int grains_gpu_upload_particles(grains_gpu_ctx* c, const grains_gpu_particles* p) {
  if (!c || !p) return GRAINS_GPU_INVALID_ARGUMENT;
  if (p->n < 0 || p->n > c->cap) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "particle count exceeds capacity");
  if (!p->id || !p->shape || !p->material || !p->radius || !p->crust || !p->mass || !p->inertia || !p->position ||
      !p->quaternion || !p->velocity || !p->omega)
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "missing particle array");
  const int64_t n = p->n;
  const int maxmat = c->cfg.max_materials > 0 ? c->cfg.max_materials : 4;
  bool basis_needed = false;
  for (int64_t i = 0; i < n; ++i) {
    if (p->shape[i] < 0 || p->shape[i] >= (int)c->shapes.size())
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "particle shape id out of range");
    if (p->material[i] < 0 || p->material[i] >= maxmat)
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "particle material out of range");
    int si = p->system ? p->system[i] : 0;
    if (si < 0 || si >= (int)c->sys.size()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "particle system out of range");
    if (c->shapes[p->shape[i]].type != GRAINS_GPU_SPHERE) basis_needed = true;
  }
  const bool nonsphere = basis_needed;
  // a basis given for spheres is kept and turned with them, as the
  // reference's transforms are (RigidBody::composeLeftByRotation)
  if (p->basis) basis_needed = true;
  // names of the particles: sorted (system, id) keys; an id appears once per system
  std::vector<std::pair<unsigned long long, int>> keyed((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const int si = p->system ? p->system[i] : 0;
    keyed[i] = {((unsigned long long)(unsigned)si << 32) | (unsigned)(p->id[i] ^ (int)0x80000000), (int)i};
  }
  std::sort(keyed.begin(), keyed.end());
  for (int64_t i = 1; i < n; ++i)
    if (keyed[i].first == keyed[i - 1].first)
      return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "a particle id appears twice in one system");
  if (c->tables_dirty) {
    if (int rc = build_tables(c)) return rc;
    c->tables_dirty = false;
  }
  c->has_basis = basis_needed;
  c->has_convex = nonsphere;
  c->all_spheres = !nonsphere;
  for (auto& s : c->sys)
    for (auto& o : s.obs)
      if (c->shapes[o.shape].type != GRAINS_GPU_BOX) c->has_convex = true;
  {
    // contact lists: 32 slots per particle for spheres, 64 when bounding
    // spheres of other shapes are listed
    const int cap_per = c->list_capacity > 0 ? c->list_capacity : (c->has_convex ? 64 : 32);
    if (!c->ccount) {
      void* q = nullptr;
      CK(cudaMalloc(&q, (size_t)c->cap * sizeof(int)));
      c->ccount = (int*)q;
    }
    if (int rc = ensure_lists(c, cap_per)) return rc;
  }
  if (basis_needed) {
    for (int k = 0; k < 2; ++k)
      if (!c->buf[k].basis) {
        void* q = nullptr;
        CK(cudaMalloc(&q, (size_t)c->cap * 9 * sizeof(double)));
        c->buf[k].basis = (double*)q;
      }
  }
  c->n = n;
  c->cur = 0;
  auto& b = c->buf[0];
  std::vector<double4> xr(n), q(n), md(n);
  std::vector<int4> meta(n);
  std::vector<int> orig(n);
  std::vector<double> basis(basis_needed ? 9 * n : 0);
  std::vector<double> vd, wd, wbfd, Id, zd;
  std::vector<float> vf, wf, wbff, If, zf;
  const bool dbl = c->precision == GRAINS_GPU_FP64;
  auto put = [&](std::vector<double>& D, std::vector<float>& Fv, int64_t i, double x, double y, double z) {
    if (dbl) {
      D[4 * i] = x; D[4 * i + 1] = y; D[4 * i + 2] = z; D[4 * i + 3] = 0;
    } else {
      Fv[4 * i] = (float)x; Fv[4 * i + 1] = (float)y; Fv[4 * i + 2] = (float)z; Fv[4 * i + 3] = 0;
    }
  };
  if (dbl) { vd.resize(4 * n); wd.resize(4 * n); wbfd.resize(4 * n); Id.resize(4 * n); zd.assign(4 * n, 0.); }
  else { vf.resize(4 * n); wf.resize(4 * n); wbff.resize(4 * n); If.resize(4 * n); zf.assign(4 * n, 0.f); }
  c->fh.id.assign(n, 0);
  c->fh.shape.assign(n, 0);
  c->fh.mass.assign(n, 0.);
  c->fh.inertia.assign(3 * n, 0.);
  c->fh.radius.assign(n, 0.);
  c->fh.density.assign(n, 0.);
  for (int64_t i = 0; i < n; ++i) {
    const ShapeHost& sh = c->shapes[p->shape[i]];
    xr[i] = make_double4(p->position[3 * i], p->position[3 * i + 1], p->position[3 * i + 2], p->radius[i]);
    Qt<double> qq{v3<double>(p->quaternion[4 * i], p->quaternion[4 * i + 1], p->quaternion[4 * i + 2]),
                  p->quaternion[4 * i + 3]};
    q[i] = make_double4(qq.v.x, qq.v.y, qq.v.z, qq.w);
    double vol = sh.type == GRAINS_GPU_SPHERE ? 4.0 * kPi * std::pow(p->radius[i], 3.) / 3.0 : sh.volume;
    double req = std::pow((0.75 / kPi) * vol, 1. / 3.);  // Component::getEquivalentSphereRadius
    md[i] = make_double4(p->mass[i], p->crust[i], req, 0.);
    meta[i] = make_int4(p->id[i], p->material[i], p->shape[i], p->system ? p->system[i] : 0);
    orig[i] = (int)i;
    c->fh.id[i] = p->id[i];
    c->fh.shape[i] = p->shape[i];
    c->fh.mass[i] = p->mass[i];
    for (int k = 0; k < 3; ++k) c->fh.inertia[3 * i + k] = p->inertia[3 * i + k];
    c->fh.radius[i] = p->radius[i];
    c->fh.density[i] = p->mass[i] / vol;
    put(vd, vf, i, p->velocity[3 * i], p->velocity[3 * i + 1], p->velocity[3 * i + 2]);
    V3<double> w = v3<double>(p->omega[3 * i], p->omega[3 * i + 1], p->omega[3 * i + 2]);
    put(wd, wf, i, w.x, w.y, w.z);
    V3<double> wbf = q_to_body(qq, w);  // ParticleKinematics::setAngularVelocity, ParticleKinematics.cpp:197-203
    put(wbfd, wbff, i, wbf.x, wbf.y, wbf.z);
    put(Id, If, i, p->inertia[3 * i], p->inertia[3 * i + 1], p->inertia[3 * i + 2]);
    if (basis_needed) {
      if (p->basis) {
        for (int k = 0; k < 9; ++k) basis[9 * i + k] = p->basis[9 * i + k];
      } else {  // rotation matrix of the quaternion
        double x = qq.v.x, y = qq.v.y, z = qq.v.z, w0 = qq.w;
        double m[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w0 * z), 2 * (x * z + w0 * y),
                       2 * (x * y + w0 * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w0 * x),
                       2 * (x * z - w0 * y), 2 * (y * z + w0 * x), 1 - 2 * (x * x + y * y)};
        for (int k = 0; k < 9; ++k) basis[9 * i + k] = m[k];
      }
    }
  }
  const size_t r4 = 4 * c->rsize;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
    if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    return 0;
  };
  int rc = 0;
  rc |= cp(b.xr, xr.data(), n * sizeof(double4));
  rc |= cp(b.q, q.data(), n * sizeof(double4));
  rc |= cp(b.md, md.data(), n * sizeof(double4));
  rc |= cp(b.meta, meta.data(), n * sizeof(int4));
  rc |= cp(b.orig, orig.data(), n * sizeof(int));
  if (basis_needed) rc |= cp(b.basis, basis.data(), 9 * n * sizeof(double));
  const void* srcs[6];
  if (dbl) {
    srcs[0] = vd.data(); srcs[1] = wd.data(); srcs[2] = wbfd.data(); srcs[3] = zd.data(); srcs[4] = zd.data();
    srcs[5] = Id.data();
  } else {
    srcs[0] = vf.data(); srcs[1] = wf.data(); srcs[2] = wbff.data(); srcs[3] = zf.data(); srcs[4] = zf.data();
    srcs[5] = If.data();
  }
  // a given torsor (a reload's force and torque) stands until the next force evaluation
  std::vector<double> Fd, Td;
  std::vector<float> Ff, Tf;
  if (p->force && p->torque) {
    if (dbl) { Fd.assign(4 * n, 0.); Td.assign(4 * n, 0.); }
    else { Ff.assign(4 * n, 0.f); Tf.assign(4 * n, 0.f); }
    for (int64_t i = 0; i < n; ++i) {
      put(Fd, Ff, i, p->force[3 * i], p->force[3 * i + 1], p->force[3 * i + 2]);
      put(Td, Tf, i, p->torque[3 * i], p->torque[3 * i + 1], p->torque[3 * i + 2]);
    }
    srcs[3] = dbl ? (const void*)Fd.data() : (const void*)Ff.data();
    srcs[4] = dbl ? (const void*)Td.data() : (const void*)Tf.data();
  }
  void* dsts[6] = {b.v, b.w, b.wbf, b.F, b.T, b.inertia};
  for (int k = 0; k < 6; ++k) rc |= cp(dsts[k], srcs[k], n * r4);
  if (rc) return rc;
  CK(cudaMemsetAsync(c->coord, 0, (size_t)c->cap * sizeof(int), c->stream));
  // tables of the reload and RawData writers
  if (!c->d_row_id) {
    void* q0 = nullptr;
    CK(cudaMalloc(&q0, (size_t)c->cap * sizeof(int)));
    c->d_row_id = (int*)q0;
    CK(cudaMalloc(&q0, (size_t)c->cap * sizeof(int)));
    c->d_row_sys = (int*)q0;
    CK(cudaMalloc(&q0, (size_t)c->cap * sizeof(unsigned long long)));
    c->d_row_keys = (unsigned long long*)q0;
    CK(cudaMalloc(&q0, (size_t)c->cap * sizeof(int)));
    c->d_key_rows = (int*)q0;
    CK(cudaMalloc(&q0, (size_t)c->cap * sizeof(RecordAttr)));
    c->d_attr = (RecordAttr*)q0;
  }
  {
    std::vector<int> rid(n), rsys(n), krow(n);
    std::vector<unsigned long long> keys(n);
    std::vector<RecordAttr> attr(n);
    for (int64_t i = 0; i < n; ++i) {
      rid[i] = p->id[i];
      rsys[i] = p->system ? p->system[i] : 0;
      keys[i] = keyed[i].first;
      krow[i] = keyed[i].second;
      // defaults: the shape's type, interior, active, a translated transform
      attr[i] = RecordAttr{p->shape[i], 0, 1, 1};
    }
    rc |= cp(c->d_row_id, rid.data(), n * sizeof(int));
    rc |= cp(c->d_row_sys, rsys.data(), n * sizeof(int));
    rc |= cp(c->d_row_keys, keys.data(), n * sizeof(unsigned long long));
    rc |= cp(c->d_key_rows, krow.data(), n * sizeof(int));
    rc |= cp(c->d_attr, attr.data(), n * sizeof(RecordAttr));
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));  // the host vectors above are pageable
  }
  c->moved = 0;
  c->fluid_corrected = 0;  // md.w (rho_f / rho_p) was uploaded as 0
  c->hydro_on = false;
  c->obs_force_valid = false;  // no force evaluation of these particles yet
  for (int k = 0; k < 2; ++k) CK(cudaMemsetAsync(c->hist_n[k], 0, (size_t)c->cap * sizeof(int), c->stream));
  for (int k = 0; k < 2; ++k)
    if (c->gdir_n[k]) CK(cudaMemsetAsync(c->gdir_n[k], 0, (size_t)c->cap * sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->stats, 0, sizeof(StatsDev), c->stream));
  c->keys_valid = false;
  c->sorted = false;
  c->pending_kick2 = false;
  c->uploaded = true;
  if (int e = sort_now(c, 1)) return e;
  return finish_call(c);
}

namespace {
// the device staging buffer of update / download: 30 doubles per particle
int ensure_stage(grains_gpu_ctx* c) {
  if (c->stage) return 0;
  void* q = nullptr;
  CK(cudaMalloc(&q, (size_t)c->cap * 30 * sizeof(double)));
  c->stage = (char*)q;
  return 0;
}
}  // namespace

// The state is permuted into upload order and widened to double on the device
// (pack_download_kernel); each requested field then goes to the caller's array
// in one copy (from pinned caller memory the copies run at the link's rate).
int grains_gpu_download_particles(grains_gpu_ctx* c, grains_gpu_particles* p) {
  if (!c || !p) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (int rc = flush_kick(c)) return rc;
  if (int rc = ensure_stage(c)) return rc;
  const int64_t n = c->n, m = std::min<int64_t>(p->n, n);
  double* d = (double*)c->stage;
  DownloadStage st{};
  st.position = p->position ? d : nullptr;
  st.quaternion = p->quaternion ? d + 3 * n : nullptr;
  st.basis = p->basis ? d + 7 * n : nullptr;
  st.velocity = p->velocity ? d + 16 * n : nullptr;
  st.omega = p->omega ? d + 19 * n : nullptr;
  st.force = p->force ? d + 22 * n : nullptr;
  st.torque = p->torque ? d + 25 * n : nullptr;
  st.coordination = p->coordination ? (int*)(d + 28 * n) : nullptr;
  st.id = p->id ? (int*)(d + 29 * n) : nullptr;
  int rc = with_args(c, [&](auto& a) { return launch_pack_download(a, c->stream, st); });
  if (rc) return fail(c, rc, "download launch failed");
  auto get = [&](void* dst, const void* src, size_t bytes) -> int {
    if (dst && bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    return 0;
  };
  rc = get(p->position, st.position, 3 * m * sizeof(double));
  rc = rc ? rc : get(p->quaternion, st.quaternion, 4 * m * sizeof(double));
  rc = rc ? rc : get(p->basis, st.basis, 9 * m * sizeof(double));
  rc = rc ? rc : get(p->velocity, st.velocity, 3 * m * sizeof(double));
  rc = rc ? rc : get(p->omega, st.omega, 3 * m * sizeof(double));
  rc = rc ? rc : get(p->force, st.force, 3 * m * sizeof(double));
  rc = rc ? rc : get(p->torque, st.torque, 3 * m * sizeof(double));
  rc = rc ? rc : get(p->coordination, st.coordination, m * sizeof(int));
  rc = rc ? rc : get(p->id, st.id, m * sizeof(int));
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  p->n = m;
  return 0;
}

// The caller's arrays go to the device staging in one copy each; the update
// kernel scatters them into the cell-ordered state.
int grains_gpu_update_particles(grains_gpu_ctx* c, const grains_gpu_particles* p) {
  if (!c || !p) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  if (p->n != c->n) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "update must cover every uploaded particle");
  if (!p->position || !p->quaternion || !p->velocity || !p->omega)
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "missing kinematic array");
  if (int rc = ensure_stage(c)) return rc;
  const int64_t n = c->n;
  if (int rc = flush_kick(c)) return rc;
  double* d = (double*)c->stage;
  const bool with_basis = c->has_basis && p->basis;
  KinematicStage st{d, d + 3 * n, d + 7 * n, d + 10 * n, with_basis ? d + 13 * n : nullptr};
  CK(cudaMemcpyAsync((void*)st.position, p->position, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync((void*)st.quaternion, p->quaternion, 4 * n * sizeof(double), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync((void*)st.velocity, p->velocity, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync((void*)st.omega, p->omega, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (with_basis)
    CK(cudaMemcpyAsync((void*)st.basis, p->basis, 9 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc = with_args(c, [&](auto& a) { return launch_update_dynamic(a, c->stream, st); });
  if (rc) return fail(c, rc, "update launch failed");
  c->keys_valid = false;
  c->sorted = false;
  if ((rc = sort_now(c, 1))) return rc;
  return finish_call(c);
}

int grains_gpu_update_particle_rows(grains_gpu_ctx* c, int64_t n_rows, const int64_t* rows,
                                    const grains_gpu_particles* p) {
  if (!c || !p || n_rows < 0 || (n_rows && !rows)) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  if (n_rows > c->n) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "more rows than particles");
  if (n_rows == 0) return 0;
  if (!p->position || !p->quaternion || !p->velocity || !p->omega)
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "missing kinematic array");
  std::vector<char> seen((size_t)c->n, 0);
  for (int64_t k = 0; k < n_rows; ++k) {
    if (rows[k] < 0 || rows[k] >= c->n) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "row out of range");
    if (seen[(size_t)rows[k]]++) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "a row appears twice");
  }
  if (int rc = ensure_stage(c)) return rc;
  if (!c->row_scratch) {  // the rows and the slot of every upload index
    void* q = nullptr;
    CK(cudaMalloc(&q, (size_t)c->cap * (sizeof(long long) + sizeof(int))));
    c->row_scratch = (char*)q;
  }
  if (int rc = flush_kick(c)) return rc;
  const int64_t m = n_rows;
  double* d = (double*)c->stage;
  const bool with_basis = c->has_basis && p->basis;
  KinematicStage st{d, d + 3 * m, d + 7 * m, d + 10 * m, with_basis ? d + 13 * m : nullptr};
  long long* drows = (long long*)c->row_scratch;
  int* slot_of = (int*)(c->row_scratch + (size_t)c->cap * sizeof(long long));
  CK(cudaMemcpyAsync(drows, rows, m * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync((void*)st.position, p->position, 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync((void*)st.quaternion, p->quaternion, 4 * m * sizeof(double), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync((void*)st.velocity, p->velocity, 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync((void*)st.omega, p->omega, 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (with_basis)
    CK(cudaMemcpyAsync((void*)st.basis, p->basis, 9 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc = with_args(c, [&](auto& a) { return launch_update_rows(a, c->stream, st, drows, m, slot_of); });
  if (rc) return fail(c, rc, "update launch failed");
  c->keys_valid = false;
  c->sorted = false;
  if ((rc = sort_now(c, 1))) return rc;
  return finish_call(c);
}

int grains_gpu_set_fluid(grains_gpu_ctx* c, double fluid_density, int32_t corrected,
                         const double* particle_density) {
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  if (!(fluid_density >= 0.) || (corrected != 0 && corrected != 1))
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "bad fluid density or correction flag");
  if (fluid_density > 0. && !particle_density)
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "particle densities are needed with a fluid");
  const int64_t n = c->n;
  std::vector<double> ratio((size_t)n, 0.);
  for (int64_t i = 0; fluid_density > 0. && i < n; ++i) {
    if (!(particle_density[i] > 0.)) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "particle density <= 0");
    ratio[(size_t)i] = fluid_density / particle_density[i];  // Particle::m_fluidDensity / m_density
  }
  if (int rc = ensure_stage(c)) return rc;
  CK(cudaMemcpyAsync(c->stage, ratio.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc = with_args(c, [&](auto& a) { return launch_set_fluid_ratio(a, c->stream, (const double*)c->stage); });
  if (rc) return fail(c, rc, "fluid set-up launch failed");
  c->fluid_corrected = fluid_density > 0. ? corrected : 0;
  if (particle_density)
    for (int64_t i = 0; i < n; ++i) c->fh.density[(size_t)i] = particle_density[i];
  drop_graphs(c);
  return finish_call(c);
}

int grains_gpu_set_velocities(grains_gpu_ctx* c, const double* velocity, const double* omega) {
  if (!c || !velocity || !omega) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  if (int rc = ensure_stage(c)) return rc;
  if (int rc = flush_kick(c)) return rc;
  const int64_t n = c->n;
  double* d = (double*)c->stage;
  CK(cudaMemcpyAsync(d, velocity, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(d + 3 * n, omega, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc = with_args(c, [&](auto& a) { return launch_set_velocities(a, c->stream, d, d + 3 * n); });
  if (rc) return fail(c, rc, "velocity launch failed");
  return finish_call(c);
}

int grains_gpu_fluid_step(grains_gpu_ctx* c, double dt_fluid, double min_dt, double max_dt, int64_t* ndt,
                          double* time) {
  if (!c || !ndt || !time || !(dt_fluid > 0.) || !(min_dt > 0.) || !(max_dt >= min_dt) || *ndt < 1)
    return GRAINS_GPU_INVALID_ARGUMENT;
  // GrainsCoupledWithFluid::Simulation (Fluid/src/GrainsCoupledWithFluid.cpp:
  // 123-135): the DEM steps of one fluid step, from the previous count
  const double dteff = std::max(std::min(max_dt, dt_fluid / double(*ndt)), min_dt);
  const int64_t m = (int64_t)(size_t)(dt_fluid / dteff);
  if (m < 1) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "fluid step shorter than the DEM step");
  *ndt = m;
  const double dt = dt_fluid / double(m);
  int64_t done = 0;
  while (done < m) {  // grains_gpu_step takes an int32 count
    const int32_t k = (int32_t)std::min<int64_t>(m - done, 1 << 30);
    if (int rc = grains_gpu_step(c, k, time, dt)) return rc;
    done += k;
  }
  return 0;
}

namespace {
// GrainsExec::doubleToString(ios::scientific, FORMAT16DIGITS, x): scientific
// with 16 digits, a zero as the stream prints it
void put_sci(std::string& o, double x) {
  char b[64];
  if (x == 0.)
    std::snprintf(b, sizeof(b), "%s", std::signbit(x) ? "-0" : "0");
  else
    std::snprintf(b, sizeof(b), "%.16e", x);
  o += b;
  o += ' ';
}
void put_int(std::string& o, long long k) {
  o += std::to_string(k);
  o += ' ';
}
}  // namespace

int grains_gpu_fluid_features(grains_gpu_ctx* c, char* buf, int64_t cap, int64_t* len) {
  if (!c || !len) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  const int64_t n = c->n;
  std::vector<double> pos(3 * n), quat(4 * n), basis(9 * n), vel(3 * n), om(3 * n);
  grains_gpu_particles p{};
  p.n = n;
  p.position = pos.data();
  p.quaternion = quat.data();
  p.basis = basis.data();
  p.velocity = vel.data();
  p.omega = om.data();
  if (int rc = grains_gpu_download_particles(c, &p)) return rc;
  std::vector<int64_t> order(n);
  for (int64_t i = 0; i < n; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return c->fh.id[a] < c->fh.id[b]; });
  // GrainsCoupledWithFluid::GrainsToFluid (Fluid/src/GrainsCoupledWithFluid.cpp:
  // 912-1120), as GrainsToBasilisk tokenises it (InterfaceGrains3DBasilisk.cpp:
  // 64-87): every token followed by one space
  std::string o;
  put_int(o, n);
  for (int64_t k = 0; k < n; ++k) {
    const int64_t i = order[k];
    const ShapeHost& sh = c->shapes[c->fh.shape[i]];
    const double* B = basis.data() + 9 * i;
    // Particle::computeInertiaTensorSpaceFixed (Particle.cpp:1798-1822):
    // Mr (I_body Mr^t), matrix products summed in index order
    double Ib[9] = {c->fh.inertia[3 * i], 0., 0., 0., c->fh.inertia[3 * i + 1], 0., 0., 0., c->fh.inertia[3 * i + 2]};
    double Bt[9], T1[9], Is[9];
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q) Bt[3 * r + q] = B[3 * q + r];
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q)
        T1[3 * r + q] = Ib[3 * r] * Bt[q] + Ib[3 * r + 1] * Bt[3 + q] + Ib[3 * r + 2] * Bt[6 + q];
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q)
        Is[3 * r + q] = B[3 * r] * T1[q] + B[3 * r + 1] * T1[3 + q] + B[3 * r + 2] * T1[6 + q];
    // corners code and envelope (Convex::getNbCorners / getEnvelope / getFaces)
    std::vector<double> env;
    const std::vector<std::vector<int>>* faces = nullptr;
    static const std::vector<std::vector<int>> box_faces = {{4, 5, 6, 7}, {5, 1, 2, 6}, {1, 0, 3, 2},
                                                            {0, 4, 7, 3}, {4, 0, 1, 5}, {3, 7, 6, 2}};
    long long corners = 1;
    if (sh.type == GRAINS_GPU_SPHERE) {
      env = {0., 0., 0.};
    } else if (sh.type == GRAINS_GPU_BOX) {  // Box::setCornersFaces (Box.cpp:92-148)
      const double ex = sh.ext.x, ey = sh.ext.y, ez = sh.ext.z;
      env = {-ex, -ey, -ez, ex, -ey, -ez, ex, -ey, ez, -ex, -ey, ez, -ex, ey, -ez, ex, ey, -ez, ex, ey, ez, -ex, ey, ez};
      faces = &box_faces;
      corners = 666;
    } else if (sh.type == GRAINS_GPU_CYLINDER) {  // Cylinder::getEnvelope (Cylinder.cpp:142-152)
      env = {0., -sh.half_height, 0., sh.radius, -sh.half_height, 0., 0., sh.half_height, 0.};
      corners = 777;
    } else {  // Polytope::getEnvelope, the polyhedron's faces
      env = sh.verts;
      faces = &sh.faces;
      corners = (long long)sh.verts.size() / 3;
    }
    put_int(o, k);
    put_int(o, corners);
    o += "P ";
    for (int t = 0; t < 3; ++t) put_sci(o, vel[3 * i + t]);
    for (int t = 0; t < 3; ++t) put_sci(o, om[3 * i + t]);
    put_sci(o, c->fh.density[i]);
    put_sci(o, c->fh.mass[i]);
    put_sci(o, Is[0]);
    put_sci(o, Is[1]);
    put_sci(o, Is[2]);
    put_sci(o, Is[4]);
    put_sci(o, Is[5]);
    put_sci(o, Is[8]);
    for (int t = 0; t < 9; ++t) put_sci(o, B[t]);
    for (int t = 0; t < 3; ++t) put_sci(o, pos[3 * i + t]);
    char rb[64];  // the circumscribed radius as the stream prints a double by default
    std::snprintf(rb, sizeof(rb), "%g", sh.type == GRAINS_GPU_SPHERE ? c->fh.radius[i] : sh.circ);
    o += rb;
    o += ' ';
    // RigidBody::writePositionInFluid (Geometry/src/RigidBody.cpp:445-497)
    const size_t np = env.size() / 3;
    put_int(o, (long long)np);
    for (size_t t = 0; t < np; ++t) {
      const double x = env[3 * t], y = env[3 * t + 1], z = env[3 * t + 2];
      put_sci(o, B[0] * x + B[1] * y + B[2] * z + pos[3 * i]);
      put_sci(o, B[3] * x + B[4] * y + B[5] * z + pos[3 * i + 1]);
      put_sci(o, B[6] * x + B[7] * y + B[8] * z + pos[3 * i + 2]);
    }
    if (faces) {
      put_int(o, (long long)faces->size());
      for (const auto& f : *faces) {
        put_int(o, (long long)f.size());
        for (int v : f) put_int(o, v);
      }
    } else {
      put_int(o, 0);
    }
  }
  *len = (int64_t)o.size() + 1;
  if (buf) {
    if (cap < *len) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "buffer too small for the features");
    std::memcpy(buf, o.c_str(), o.size() + 1);
  }
  return 0;
}

int grains_gpu_set_hydro_forces(grains_gpu_ctx* c, const double* force, const double* torque) {
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  const bool on = force || torque;
  if (on) {
    if (!c->d_hydro) {
      void* q = nullptr;
      CK(cudaMalloc(&q, (size_t)c->cap * 6 * sizeof(double)));
      c->d_hydro = (double*)q;
    }
    const int64_t n = c->n;
    std::vector<double> h((size_t)n * 6, 0.);
    for (int64_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) {
        if (force) h[6 * i + k] = force[3 * i + k];
        if (torque) h[6 * i + 3 + k] = torque[3 * i + k];
      }
    CK(cudaMemcpyAsync(c->d_hydro, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));  // h is pageable
  }
  if (on != c->hydro_on) drop_graphs(c);
  c->hydro_on = on;
  return 0;
}

// ---- the fluid solvers' C interface (InterfaceGrains3DBasilisk.h:12-30) ----
// The reference keeps one coupled simulation in a static (InterfaceGrains3DBasilisk
// .cpp:16) built by Init_Grains from its XML and reload files; here the caller
// sets up a context through the grains_gpu calls and attaches it, and the
// interface drives that context.
namespace {
struct BasiliskState {
  grains_gpu_ctx* ctx = nullptr;
  double min_dt = 0., max_dt = 0.;
  int64_t ndt = 1;
  double time = 0.;
  int cycle = 0;
};
BasiliskState g_basilisk;

[[noreturn]] void basilisk_abort(const char* where, const std::string& why) {
  // the reference ends the run on a set-up or simulation error (grainsAbort)
  std::fprintf(stderr, "%s: %s\n", where, why.c_str());
  std::exit(1);
}
void basilisk_check(const char* where, int rc) {
  if (rc) {
    char m[512] = {0};
    if (g_basilisk.ctx) grains_gpu_last_error(g_basilisk.ctx, m, sizeof(m));
    basilisk_abort(where, m[0] ? m : "grains_gpu error");
  }
}
grains_gpu_ctx* basilisk_ctx(const char* where) {
  if (!g_basilisk.ctx) basilisk_abort(where, "no context attached (grains_gpu_basilisk_attach)");
  return g_basilisk.ctx;
}
}  // namespace

int grains_gpu_basilisk_attach(grains_gpu_ctx* c, double min_dt, double max_dt, int64_t ndt) {
  if (!c || !(min_dt > 0.) || !(max_dt >= min_dt) || ndt < 1) return GRAINS_GPU_INVALID_ARGUMENT;
  g_basilisk = BasiliskState();
  g_basilisk.ctx = c;
  g_basilisk.min_dt = min_dt;
  g_basilisk.max_dt = max_dt;
  g_basilisk.ndt = ndt;
  return 0;
}

void Init_Grains(char const* inputfile, double fluid_rho, const bool b_restart, const bool b_fluidcorrectedacc) {
  (void)inputfile;
  (void)b_restart;
  grains_gpu_ctx* c = basilisk_ctx("Init_Grains");
  // GrainsCoupledWithFluid(fluid_density) and setFluidCorrectedAcceleration
  // (InterfaceGrains3DBasilisk.cpp:28-48), then the leapfrog start
  basilisk_check("Init_Grains", grains_gpu_set_fluid(c, fluid_rho, b_fluidcorrectedacc ? 1 : 0, c->fh.density.data()));
  basilisk_check("Init_Grains", grains_gpu_initialize_leapfrog(c, g_basilisk.time, g_basilisk.min_dt));
}

void Simu_Grains(const double dt_fluid) {
  grains_gpu_ctx* c = basilisk_ctx("Simu_Grains");
  basilisk_check("Simu_Grains", grains_gpu_fluid_step(c, dt_fluid, g_basilisk.min_dt, g_basilisk.max_dt,
                                                      &g_basilisk.ndt, &g_basilisk.time));
}

char* GrainsToBasilisk(int* pstrsize) {
  grains_gpu_ctx* c = basilisk_ctx("GrainsToBasilisk");
  int64_t len = 0;
  basilisk_check("GrainsToBasilisk", grains_gpu_fluid_features(c, nullptr, 0, &len));
  char* out = (char*)std::malloc((size_t)len);
  if (!out) basilisk_abort("GrainsToBasilisk", "out of host memory");
  basilisk_check("GrainsToBasilisk", grains_gpu_fluid_features(c, out, len, &len));
  if (pstrsize) *pstrsize = (int)len;
  return out;
}

void SetInitialTime(double tinit) { g_basilisk.time = tinit; }

void SetInitialCycleNumber(int cycle0) { g_basilisk.cycle = cycle0; }

void SaveResults_Grains() { ++g_basilisk.cycle; }

void checkParaviewPostProcessing_Grains(char* solid_resDir) { (void)solid_resDir; }

void UpdateVelocityGrains(double** arrayv, const int m) {
  grains_gpu_ctx* c = basilisk_ctx("UpdateVelocityGrains");
  const int64_t n = c->n;
  if (m != n) basilisk_abort("UpdateVelocityGrains", "the fluid holds another number of particles");
  std::vector<double> pos(3 * n), quat(4 * n), vel(3 * n), om(3 * n);
  grains_gpu_particles p{};
  p.n = n;
  p.position = pos.data();
  p.quaternion = quat.data();
  p.velocity = vel.data();
  p.omega = om.data();
  basilisk_check("UpdateVelocityGrains", grains_gpu_download_particles(c, &p));
  // GrainsCoupledWithFluid::updateParticlesVelocity (GrainsCoupledWithFluid.cpp:
  // 1126-1185): row k of the fluid's array is the particle of the k-th id
  std::vector<int64_t> order(n);
  for (int64_t i = 0; i < n; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return c->fh.id[a] < c->fh.id[b]; });
  for (int64_t k = 0; k < n; ++k)
    for (int t = 0; t < 3; ++t) {
      vel[3 * order[k] + t] = arrayv[k][t];
      om[3 * order[k] + t] = arrayv[k][3 + t];
    }
  basilisk_check("UpdateVelocityGrains", grains_gpu_set_velocities(c, vel.data(), om.data()));
}

void NumberOfRigidBodiesInBasilisk(size_t* nparticles, size_t* nobstacles) {
  grains_gpu_ctx* c = basilisk_ctx("NumberOfRigidBodiesInBasilisk");
  *nparticles = (size_t)c->n;
  *nobstacles = 0;
}

int grains_gpu_upload_contact_memory(grains_gpu_ctx* c, const grains_gpu_contact_memory* m) {
  if (!c || !m) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  const int64_t n = c->n;
  std::vector<int4> meta(n);
  std::vector<int> orig(n);
  auto& b = c->buf[c->cur];
  CK(cudaMemcpyAsync(meta.data(), b.meta, n * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(orig.data(), b.orig, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::map<std::pair<int, int>, int> row_of;  // (system, id) -> row (upload index)
  for (int64_t s = 0; s < n; ++s) row_of[std::make_pair(meta[s].w, meta[s].x)] = orig[s];
  std::vector<int> sys_of_row(n);
  for (int64_t s = 0; s < n; ++s) sys_of_row[orig[s]] = meta[s].w;
  const int H = c->hist_cap;
  std::vector<int> cnt(n, 0);
  const bool dbl = c->precision == GRAINS_GPU_FP64;
  std::vector<HistEntry<double>> hd(dbl ? n * H : 0);
  std::vector<HistEntry<float>> hf(dbl ? 0 : n * H);
  for (int64_t k = 0; k < m->n; ++k) {
    // find the owner row in any system holding that id (ids are unique per system;
    // the owner's system decides)
    int owner = m->owner[k], other = m->other[k];
    const size_t s0 = m->system ? (size_t)std::max(0, m->system[k]) : 0;
    const size_t s1 = m->system ? std::min(s0 + 1, c->sys.size()) : c->sys.size();
    for (size_t si = s0; si < s1; ++si) {
      auto it = row_of.find(std::make_pair((int)si, owner));
      if (it == row_of.end()) continue;
      int row = it->second;
      int flags = 0, key = other;
      auto jt = row_of.find(std::make_pair((int)si, other));
      if (jt == row_of.end()) {  // an obstacle of the system
        const SysHost& s = c->sys[si];
        int found = -1;
        for (size_t oi = 0; oi < s.obs.size(); ++oi)
          if (s.obs[oi].id == other) found = (int)oi;
        if (found < 0) break;
        flags = 1;
        key = found;
      } else if (!(owner < other)) {
        break;  // the lower id holds the pair's memory
      }
      if (cnt[row] >= H) return fail(c, GRAINS_GPU_HISTORY_FULL, "contact memory row full at upload");
      size_t e = (size_t)row * H + cnt[row]++;
      if (dbl) {
        HistEntry<double>& x = hd[e];
        x.other = key; x.flags = flags;
        for (int t = 0; t < 3; ++t) {
          x.kd[t] = m->kdelta[3 * k + t]; x.n[t] = m->prev_normal[3 * k + t]; x.sp[t] = m->spring_torque[3 * k + t];
        }
      } else {
        HistEntry<float>& x = hf[e];
        x.other = key; x.flags = flags;
        for (int t = 0; t < 3; ++t) {
          x.kd[t] = (float)m->kdelta[3 * k + t]; x.n[t] = (float)m->prev_normal[3 * k + t];
          x.sp[t] = (float)m->spring_torque[3 * k + t];
        }
      }
      break;
    }
  }
  const size_t esz = dbl ? sizeof(HistEntry<double>) : sizeof(HistEntry<float>);
  CK(cudaMemcpyAsync(c->hist[c->hcur], dbl ? (void*)hd.data() : (void*)hf.data(), (size_t)n * H * esz,
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->hist_n[c->hcur], cnt.data(), n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int grains_gpu_download_contact_memory(grains_gpu_ctx* c, grains_gpu_contact_memory* m) {
  if (!c || !m) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  const int64_t n = c->n;
  const int H = c->hist_cap;
  const bool dbl = c->precision == GRAINS_GPU_FP64;
  const size_t esz = dbl ? sizeof(HistEntry<double>) : sizeof(HistEntry<float>);
  std::vector<char> h((size_t)n * H * esz);
  std::vector<int> cnt(n);
  std::vector<int4> meta(n);
  std::vector<int> orig(n);
  auto& b = c->buf[c->cur];
  CK(cudaMemcpyAsync(h.data(), c->hist[c->hcur], h.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(cnt.data(), c->hist_n[c->hcur], n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(meta.data(), b.meta, n * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(orig.data(), b.orig, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<int> id_of_row(n), sys_of_row(n);
  for (int64_t s = 0; s < n; ++s) {
    id_of_row[orig[s]] = meta[s].x;
    sys_of_row[orig[s]] = meta[s].w;
  }
  int64_t k = 0, cap = m->n;
  int cur_sys = 0;
  auto emit = [&](int owner, int other, const double* kd, const double* nn, const double* sp, double sign) {
    if (k < cap) {
      m->owner[k] = owner;
      m->other[k] = other;
      if (m->system) m->system[k] = cur_sys;
      for (int t = 0; t < 3; ++t) {
        m->kdelta[3 * k + t] = sign * kd[t];
        m->prev_normal[3 * k + t] = sign * nn[t];
        m->spring_torque[3 * k + t] = sign * sp[t];
      }
    }
    ++k;
  };
  for (int64_t row = 0; row < n; ++row) {
    for (int e = 0; e < cnt[row]; ++e) {
      double kd[3], nn[3], sp[3];
      int other, flags;
      if (dbl) {
        const HistEntry<double>& x = ((const HistEntry<double>*)h.data())[(size_t)row * H + e];
        other = x.other; flags = x.flags;
        for (int t = 0; t < 3; ++t) { kd[t] = x.kd[t]; nn[t] = x.n[t]; sp[t] = x.sp[t]; }
      } else {
        const HistEntry<float>& x = ((const HistEntry<float>*)h.data())[(size_t)row * H + e];
        other = x.other; flags = x.flags;
        for (int t = 0; t < 3; ++t) { kd[t] = x.kd[t]; nn[t] = x.n[t]; sp[t] = x.sp[t]; }
      }
      int owner = id_of_row[row];
      cur_sys = sys_of_row[row];
      if (flags & 1) {
        const SysHost& s = c->sys[sys_of_row[row]];
        int oid = (other >= 0 && other < (int)s.obs.size()) ? s.obs[other].id : other;
        emit(owner, oid, kd, nn, sp, 1.);
        emit(oid, owner, kd, nn, sp, -1.);
      } else {
        emit(owner, other, kd, nn, sp, 1.);
        emit(other, owner, kd, nn, sp, -1.);  // mirrored entry (HookeMemoryContactForceModel.cpp:191-192)
      }
    }
  }
  m->n = k;
  return k > cap ? fail(c, GRAINS_GPU_PAIR_OVERFLOW, "contact memory buffer too small") : 0;
}

int grains_gpu_download_obstacles(grains_gpu_ctx* c, int32_t system, int32_t n, double* t) {
  if (!c || !t) return GRAINS_GPU_INVALID_ARGUMENT;
  if (system < 0 || system >= (int)c->sys.size()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "bad system");
  const SysHost& s = c->sys[system];
  if (!c->uploaded || c->h_sys.empty()) {
    for (int i = 0; i < n && i < (int)s.obs.size(); ++i)
      for (int k = 0; k < 12; ++k) t[12 * i + k] = s.obs[i].transform[k];
    return 0;
  }
  const int first = c->h_sys[system].obs_offset, cnt = c->h_sys[system].n_obs;
  std::vector<ObstacleDev> h(cnt);
  if (cnt) CK(cudaMemcpyAsync(h.data(), c->d_obs + first, cnt * sizeof(ObstacleDev), cudaMemcpyDeviceToHost,
                              c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n && i < cnt; ++i) {
    for (int k = 0; k < 9; ++k) t[12 * i + k] = h[i].b[k];
    for (int k = 0; k < 3; ++k) t[12 * i + 9 + k] = h[i].o[k];
  }
  return 0;
}

int grains_gpu_compute_forces(grains_gpu_ctx* c, double time, double dt) {
  (void)time;
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (int rc = flush_kick(c)) return rc;
  CK(cudaMemsetAsync(c->pairs_n, 0, sizeof(unsigned long long), c->stream));
  if (int rc = forces_now(c, dt, 1)) return rc;
  return finish_call(c);
}

int grains_gpu_move(grains_gpu_ctx* c, double time, double dt_v, double dt_x) {
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (int rc = flush_kick(c)) return rc;
  if (!c->sorted) {
    if (int rc = sort_now(c, 1)) return rc;
  }
  int rc = with_args(c, [&](auto& a) { return launch_kick_move(a, c->stream, 0, 0., 1, dt_v, dt_x); });
  if (rc) return fail(c, rc, "move launch failed");
  c->moved = 1;
  c->keys_valid = true;
  c->sorted = false;
  if ((rc = move_obstacles(c, dt_x, 1, time))) return rc;
  return finish_call(c);
}

int grains_gpu_link_update(grains_gpu_ctx* c, double time, double dt) {
  (void)time;
  (void)dt;
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (!c->sorted)
    if (int rc = sort_now(c, 1)) return rc;
  return finish_call(c);
}

int grains_gpu_advance_velocity(grains_gpu_ctx* c, double time, double dt_v) {
  (void)time;
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (int rc = flush_kick(c)) return rc;
  int rc = with_args(c, [&](auto& a) { return launch_kick_move(a, c->stream, 1, dt_v, 0, 0., 0.); });
  if (rc) return fail(c, rc, "advance-velocity launch failed");
  return finish_call(c);
}

int grains_gpu_initialize_leapfrog(grains_gpu_ctx* c, double time, double dt) {
  if (int rc = grains_gpu_compute_forces(c, time, dt)) return rc;
  int rc = with_args(c, [&](auto& a) { return launch_zero_kdelta(a, c->stream); });
  if (rc) return fail(c, rc, "zero-kdelta launch failed");
  return finish_call(c);
}

int grains_gpu_step(grains_gpu_ctx* c, int32_t n_steps, double* time, double dt) {
  if (!c || !time || n_steps < 0 || !(dt > 0)) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (n_steps == 0) return 0;
  c->moved = 1;
  if (!c->sorted)
    if (int rc = sort_now(c, 1)) return rc;
  // step 1 moves (finishing any pending half kick); steps 1..n-1 end with
  // the kick that also moves to the next step; step n ends with a force
  // evaluation and leaves its second half kick pending
  if (int rc = first_move(c, dt, *time)) return rc;
  int middle = n_steps - 1;
  // the persistent kernel carries Johnson's GJK only: the signed-volume one runs from the graphs
  // (force-driven obstacles need the contact-force sums between the phases:
  // launched steps only)
  if (c->persistent && middle > 0 && !(c->gjk_sv && c->has_convex) && c->n_force_obs == 0) {
    if (int rc = persistent_middle_steps(c, middle, dt)) return rc;
    middle = 0;
  }
  // a graph holds G middle steps starting right after a gather: G = the gather
  // period, doubled when odd, so that the contact-memory buffers (swapped every
  // step) come back; (cur, hcur) then select the graph
  const int G = c->gather_every % 2 ? 2 * c->gather_every : c->gather_every;
  while (middle > 0 && c->since_gather % c->gather_every != 0) {
    if (int rc = middle_step(c, dt)) return rc;
    --middle;
  }
  while (middle >= G) {
    const int slot = 2 * c->cur + c->hcur;
    if (!c->graph[slot] || c->graph_dt[slot] != dt) {
      if (c->graph[slot]) {
        cudaGraphExecDestroy(c->graph[slot]);
        c->graph[slot] = nullptr;
      }
      const int cur0 = c->cur, h0 = c->hcur;
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      const int sg0 = c->since_gather;
      int rc = 0;
      for (int k = 0; k < G && !rc; ++k) rc = middle_step(c, dt);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      c->cur = cur0;  // capturing does not execute: restore the buffer selection
      c->hcur = h0;
      c->since_gather = sg0;
      c->keys_valid = true;
      c->sorted = false;
      if (rc) return rc;
      if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&c->graph[slot], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
      c->graph_dt[slot] = dt;
    }
    CK(cudaGraphLaunch(c->graph[slot], c->stream));
    for (int k = 0; k < G; ++k) {  // the buffer selection the graph leaves
      if (c->since_gather + 1 >= c->gather_every) {
        c->cur = 1 - c->cur;
        c->since_gather = 0;
      } else {
        ++c->since_gather;
      }
      c->hcur = 1 - c->hcur;
    }
    middle -= G;
  }
  while (middle-- > 0)
    if (int rc = middle_step(c, dt)) return rc;
  if (int rc = last_step(c, dt)) return rc;
  for (int k = 0; k < n_steps; ++k) *time += dt;  // Grains::Simulation's clock
  c->steps_done += n_steps;
  return 0;
}

int grains_gpu_synchronize(grains_gpu_ctx* c) {
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  return finish_call(c);
}

int grains_gpu_get_candidate_pairs(grains_gpu_ctx* c, int32_t system, int32_t include_obstacles, int64_t cap,
                                   int32_t* pairs, int64_t* n) {
  if (!c || !n || (cap > 0 && !pairs)) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (!c->sorted)
    if (int rc = sort_now(c, 1)) return rc;
  if (!c->cand) {
    void* q = nullptr;
    c->cand_cap = (int)std::min<int64_t>(48 * c->cap + 4096, (int64_t)1 << 30);
    CK(cudaMalloc(&q, 2 * (size_t)c->cand_cap * sizeof(int)));
    c->cand = (int*)q;
    CK(cudaMalloc(&q, sizeof(unsigned long long)));
    c->cand_n = (unsigned long long*)q;
  }
  CK(cudaMemsetAsync(c->cand_n, 0, sizeof(unsigned long long), c->stream));
  int rc = with_args(c, [&](auto& a) {
    return launch_candidate_pairs(a, c->stream, system, include_obstacles, c->cand, c->cand_cap, c->cand_n);
  });
  if (rc) return fail(c, rc, "candidate pair launch failed");
  unsigned long long cnt = 0;
  CK(cudaMemcpyAsync(&cnt, c->cand_n, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (cnt > (unsigned long long)c->cand_cap) return fail(c, GRAINS_GPU_PAIR_OVERFLOW, "device pair buffer too small");
  std::vector<int> h(2 * cnt);
  if (cnt) CK(cudaMemcpy(h.data(), c->cand, 2 * cnt * sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<std::pair<int, int>> pp, po;
  for (size_t k = 0; k < cnt; ++k) {
    // particle pairs were emitted as (lower, higher); obstacle pairs as (particle, obstacle id)
    bool is_obs = false;
    const SysHost& s = c->sys[system];
    for (auto& o : s.obs)
      if (o.id == h[2 * k + 1]) is_obs = true;
    (is_obs ? po : pp).push_back(std::make_pair(h[2 * k], h[2 * k + 1]));
  }
  std::sort(pp.begin(), pp.end());
  std::sort(po.begin(), po.end());
  pp.insert(pp.end(), po.begin(), po.end());
  *n = (int64_t)pp.size();
  for (int64_t k = 0; k < (int64_t)pp.size() && k < cap; ++k) {
    pairs[2 * k] = pp[k].first;
    pairs[2 * k + 1] = pp[k].second;
  }
  return (int64_t)pp.size() > cap ? fail(c, GRAINS_GPU_PAIR_OVERFLOW, "pair buffer too small") : 0;
}

namespace {
// The diagnostic contact pairs of `system` from the last force evaluation,
// sorted by (id, id): indices into the device lists
int system_pairs(grains_gpu_ctx* c, int32_t system, std::vector<int>& h, std::vector<double>* f,
                 std::vector<size_t>& idx) {
  if (system < 0 || system >= (int)c->sys.size()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "bad system index");
  unsigned long long cnt = 0;
  CK(cudaMemcpyAsync(&cnt, c->pairs_n, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (cnt > (unsigned long long)c->pairs_cap) return fail(c, GRAINS_GPU_PAIR_OVERFLOW, "device pair buffer too small");
  h.assign(2 * cnt, 0);
  std::vector<int> sy(cnt);
  if (f) f->assign(3 * cnt, 0.);
  if (cnt) {
    CK(cudaMemcpy(h.data(), c->pairs, 2 * cnt * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sy.data(), c->pair_sys, cnt * sizeof(int), cudaMemcpyDeviceToHost));
    if (f) CK(cudaMemcpy(f->data(), c->pair_force, 3 * cnt * sizeof(double), cudaMemcpyDeviceToHost));
  }
  idx.clear();
  for (size_t k = 0; k < cnt; ++k)
    if (sy[k] == system) idx.push_back(k);
  std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) {
    return std::make_pair(h[2 * x], h[2 * x + 1]) < std::make_pair(h[2 * y], h[2 * y + 1]);
  });
  return 0;
}
}  // namespace

int grains_gpu_get_contact_pairs(grains_gpu_ctx* c, int32_t system, int64_t cap, int32_t* pairs, int64_t* n) {
  if (!c || !n || (cap > 0 && !pairs)) return GRAINS_GPU_INVALID_ARGUMENT;
  std::vector<int> h;
  std::vector<size_t> idx;
  if (int rc = system_pairs(c, system, h, nullptr, idx)) return rc;
  *n = (int64_t)idx.size();
  for (int64_t k = 0; k < (int64_t)idx.size() && k < cap; ++k) {
    pairs[2 * k] = h[2 * idx[k]];
    pairs[2 * k + 1] = h[2 * idx[k] + 1];
  }
  return (int64_t)idx.size() > cap ? fail(c, GRAINS_GPU_PAIR_OVERFLOW, "pair buffer too small") : 0;
}

int grains_gpu_get_contact_forces(grains_gpu_ctx* c, int32_t system, int64_t cap, int32_t* pairs, double* forces,
                                  int64_t* n) {
  if (!c || !n || (cap > 0 && (!pairs || !forces))) return GRAINS_GPU_INVALID_ARGUMENT;
  std::vector<int> h;
  std::vector<double> f;
  std::vector<size_t> idx;
  if (int rc = system_pairs(c, system, h, &f, idx)) return rc;
  *n = (int64_t)idx.size();
  for (int64_t k = 0; k < (int64_t)idx.size() && k < cap; ++k) {
    pairs[2 * k] = h[2 * idx[k]];
    pairs[2 * k + 1] = h[2 * idx[k] + 1];
    for (int d = 0; d < 3; ++d) forces[3 * k + d] = f[3 * idx[k] + d];
  }
  return (int64_t)idx.size() > cap ? fail(c, GRAINS_GPU_PAIR_OVERFLOW, "pair buffer too small") : 0;
}

int grains_gpu_get_stats(grains_gpu_ctx* c, grains_gpu_stats* st) {
  if (!c || !st) return GRAINS_GPU_INVALID_ARGUMENT;
  StatsDev d{};
  CK(cudaMemcpyAsync(&d, c->stats, sizeof(d), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::memset(st, 0, sizeof(*st));
  st->n_particles = c->n;
  st->n_candidate_pairs = (int64_t)d.n_cand;
  st->n_obstacle_candidates = (int64_t)d.n_obs_cand;
  st->n_contacts = (int64_t)d.n_contacts;
  st->n_obstacle_contacts = (int64_t)d.n_obs_contacts;
  st->n_gjk_calls = (int64_t)d.n_gjk_calls;
  st->n_gjk_iterations = (int64_t)d.n_gjk_iters;
  double omax;
  std::memcpy(&omax, &d.overlap_max_bits, sizeof(double));
  st->overlap_max = omax;
  st->overlap_sum = d.overlap_sum;
  st->n_steps_done = c->steps_done;
  st->status = d.status;
  const double met = double(d.n_contacts + d.n_obs_contacts);
  st->overlap_mean = met > 0. ? d.overlap_sum / met : 0.;
  st->gjk_iterations_mean = d.n_gjk_calls ? double(d.n_gjk_iters) / double(d.n_gjk_calls) : 0.;
  return 0;
}

int grains_gpu_reset_stats(grains_gpu_ctx* c) {
  if (!c) return GRAINS_GPU_INVALID_ARGUMENT;
  CK(cudaMemsetAsync(c->stats, 0, sizeof(StatsDev), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int grains_gpu_set_barrier_test(grains_gpu_ctx* c, int64_t polls, int32_t skip_block) {
  if (!c || polls < 1) return GRAINS_GPU_INVALID_ARGUMENT;
  c->barrier_polls = polls;
  c->barrier_skip_block = skip_block < 0 ? -1 : skip_block;
  return 0;
}

int grains_gpu_launches_per_step(grains_gpu_ctx* c, int64_t* launches) {
  if (!c || !launches) return GRAINS_GPU_INVALID_ARGUMENT;
  // a middle step: scan_tiles, scatter, cell_sort, contacts,
  // (the GJK kernel of convex scenarios,) pairs, sums with the kick, and the
  // obstacle move when obstacles move; the gather runs one step in
  // gather_every on top
  *launches = launches_per_middle_step() + (c->has_convex && !c->gjk_sv ? 3 : 0) + (c->n_moving > 0 ? 1 : 0) +
               (c->n_force_obs > 0 ? 1 : 0);
  return 0;
}

int grains_gpu_profile_kernels(grains_gpu_ctx* c, int32_t n_steps, double* time, double dt, char* names,
                               size_t cap, double* ms, int64_t* launches, int32_t max_kernels, int32_t* n_kernels) {
  if (!c || !time || !names || !ms || !launches || !n_kernels || max_kernels < 4)
    return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (n_steps < 2) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "profile at least 2 steps");
  if (!c->sorted)
    if (int rc = sort_now(c, 1)) return rc;
  // same schedule as grains_gpu_step, uncaptured, with events around each phase
  cudaEvent_t ev[7];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  double acc[6] = {0, 0, 0, 0, 0, 0};  // first move, sort+gather, contact lists, pair law, sums with the kick, obstacle moves
  int64_t cnt[6] = {0, 0, 0, 0, 0, 0};
  CK(cudaEventRecord(ev[0], c->stream));
  if (int rc = first_move(c, dt, *time)) return rc;
  CK(cudaEventRecord(ev[1], c->stream));
  CK(cudaEventSynchronize(ev[1]));
  float m = 0;
  cudaEventElapsedTime(&m, ev[0], ev[1]);
  acc[0] += m;
  cnt[0] += 1;
  for (int k = 0; k < n_steps; ++k) {
    const bool last = (k == n_steps - 1);
    CK(cudaEventRecord(ev[1], c->stream));
    if (int rc = last ? sort_now(c, 0) : sort_for_step(c)) return rc;
    CK(cudaEventRecord(ev[2], c->stream));
    if (int rc = forces_now(c, dt, 0, 1)) return rc;
    CK(cudaEventRecord(ev[3], c->stream));
    if (int rc = forces_now(c, dt, 0, 2)) return rc;
    CK(cudaEventRecord(ev[4], c->stream));
    if (int rc = forces_now(c, dt, 0, 4, last ? 0 : 1)) return rc;  // sums with the kick (a middle step)
    CK(cudaEventRecord(ev[5], c->stream));
    if (!last) {
      c->keys_valid = true;
      c->sorted = false;
      if (int rc2 = move_obstacles(c, dt)) return rc2;
    }
    CK(cudaEventRecord(ev[6], c->stream));
    CK(cudaEventSynchronize(ev[6]));
    float t[5] = {0, 0, 0, 0, 0};
    for (int q = 0; q < 5; ++q) cudaEventElapsedTime(&t[q], ev[1 + q], ev[2 + q]);
    for (int q = 0; q < 5; ++q) acc[1 + q] += t[q];
    cnt[1] += 3;  // scan_tiles, scatter, cell_sort (+ a gather one step in gather_every)
    cnt[2] += 1;
    cnt[3] += 1;
    cnt[4] += 1;
  }
  c->pending_kick2 = true;
  c->pending_dt = 0.5 * dt;
  for (auto& e : ev) cudaEventDestroy(e);
  for (int k = 0; k < n_steps; ++k) *time += dt;
  c->steps_done += n_steps;
  std::snprintf(names, cap, "first_move\nsort_gather\ncontacts\npairs\nsums_kick\nobstacle_move");
  const int nk = max_kernels < 6 ? max_kernels : 6;
  for (int k = 0; k < nk; ++k) {
    ms[k] = acc[k];
    launches[k] = cnt[k];
  }
  *n_kernels = nk;
  return finish_call(c);
}

int grains_gpu_shape_properties(int32_t type, const double* params, int32_t n, double* volume, double* circ,
                                double inertia[3]) {
  if (!params || !volume || !circ || !inertia) return GRAINS_GPU_INVALID_ARGUMENT;
  ShapeHost s;
  std::string err;
  if (int rc = build_shape(type, params, n, s, err)) return rc;
  *volume = s.volume;
  *circ = s.circ;
  for (int i = 0; i < 3; ++i) inertia[i] = s.inertia[i];
  return 0;
}


// ---- tuning ------------------------------------------------------------------
int grains_gpu_get_tuning(const grains_gpu_ctx* c, grains_gpu_tuning* t) {
  if (!c || !t) return GRAINS_GPU_INVALID_ARGUMENT;
  std::memset(t, 0, sizeof(*t));
  t->cell_factor = c->cell_factor;
  t->contacts_block = c->contacts_block;
  t->forces_block = c->forces_block;
  t->list_capacity = c->list_capacity > 0 ? c->list_capacity : c->clist_cap;
  t->gather_every = c->gather_every;
  t->persistent = c->persistent;
  return 0;
}

int grains_gpu_set_tuning(grains_gpu_ctx* c, const grains_gpu_tuning* t) {
  if (!c || !t) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!(t->cell_factor >= 1.0 && t->cell_factor <= 4.0) || t->contacts_block < 32 || t->contacts_block > 256 ||
      t->contacts_block % 32 || t->forces_block < 32 || t->forces_block > 128 || t->forces_block % 32 ||
      (t->list_capacity != 0 && (t->list_capacity < 8 || t->list_capacity > 256 || t->list_capacity % 4)) || t->gather_every < 1 ||
      t->gather_every > 64)
    return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "tuning out of range");
  const bool regrid = t->cell_factor != c->cell_factor;
  c->cell_factor = t->cell_factor;
  c->contacts_block = t->contacts_block;
  c->forces_block = t->forces_block;
  c->list_capacity = t->list_capacity;
  c->gather_every = t->gather_every;
  c->persistent = t->persistent ? 1 : 0;
  c->pblocks = 0;  // the block count follows the kernel variant (convex or not)
  if (c->psums) {
    cudaFree(c->psums);
    c->psums = nullptr;
  }
  for (int k = 0; k < 4; ++k)  // launch shapes and the gather period are baked into the step graphs
    if (c->graph[k]) {
      cudaGraphExecDestroy(c->graph[k]);
      c->graph[k] = nullptr;
    }
  for (auto& s : c->sys)
    if (s.has_domain)
      if (int rc = apply_grid(c, s)) return rc;
  if (!c->uploaded) {
    c->tables_dirty = true;
    return 0;
  }
  if (regrid) {
    // rebuild the cell tables for the new grid; moving obstacles keep their
    // current poses and velocities
    std::vector<ObstacleDev> live(c->h_obs.size());
    std::vector<int> flags(2 * c->sys.size());
    std::vector<double> pid(c->d_force_pid ? c->sys.size() * kForcePidWords : 0);
    if (!live.empty()) {
      CK(cudaMemcpyAsync(live.data(), c->d_obs, live.size() * sizeof(ObstacleDev), cudaMemcpyDeviceToHost,
                         c->stream));
      CK(cudaMemcpyAsync(flags.data(), c->d_load_flags, flags.size() * sizeof(int), cudaMemcpyDeviceToHost,
                         c->stream));
      if (!pid.empty())
        CK(cudaMemcpyAsync(pid.data(), c->d_force_pid, pid.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
    if (int rc = build_tables(c)) return rc;
    if (!live.empty()) {
      CK(cudaMemcpyAsync(c->d_obs, live.data(), live.size() * sizeof(ObstacleDev), cudaMemcpyHostToDevice,
                         c->stream));
      CK(cudaMemcpyAsync(c->d_load_flags, flags.data(), flags.size() * sizeof(int), cudaMemcpyHostToDevice,
                         c->stream));
      if (!pid.empty() && c->d_force_pid)
        CK(cudaMemcpyAsync(c->d_force_pid, pid.data(), pid.size() * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
    c->sorted = false;
    c->keys_valid = false;
    c->obs_force_valid = false;  // the contact lists are rebuilt with the next force evaluation
  }
  const int cap_per = c->list_capacity > 0 ? c->list_capacity : (c->has_convex ? 64 : 32);
  CK(cudaStreamSynchronize(c->stream));
  if (int rc = ensure_lists(c, cap_per)) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

namespace {
// exact device copy of the dynamic state of a context (particles, contact
// memory, obstacle poses, clock), for trials that must start from it
struct Snapshot {
  std::vector<std::pair<void*, size_t>> bufs;  // (device copy, bytes), in the order of fields()
  int cur = 0, hcur = 0, since_gather = 0;
  bool pending = false;
  double pending_dt = 0.;
  int64_t steps_done = 0;
};

std::vector<std::pair<void*, size_t>> snapshot_fields(grains_gpu_ctx* c, int cur, int hcur) {
  const size_t n = (size_t)c->n, r4 = 4 * c->rsize;
  auto& b = c->buf[cur];
  const size_t hsz = c->precision == GRAINS_GPU_FP64 ? sizeof(HistEntry<double>) : sizeof(HistEntry<float>);
  std::vector<std::pair<void*, size_t>> f = {
      {b.xr, n * sizeof(double4)}, {b.q, n * sizeof(double4)}, {b.v, n * r4}, {b.w, n * r4},
      {b.wbf, n * r4}, {b.F, n * r4}, {b.T, n * r4}, {b.inertia, n * r4},
      {b.md, n * sizeof(double4)}, {b.meta, n * sizeof(int4)}, {b.orig, n * sizeof(int)},
      {c->hist[hcur], n * c->hist_cap * hsz}, {c->hist_n[hcur], n * sizeof(int)},
      {c->clock, sizeof(double)}};
  if (c->has_basis) f.push_back({b.basis, 9 * n * sizeof(double)});
  if (!c->h_obs.empty()) f.push_back({c->d_obs, c->h_obs.size() * sizeof(ObstacleDev)});
  if (!c->h_obs.empty()) f.push_back({c->d_load_flags, 2 * c->sys.size() * sizeof(int)});
  if (c->d_force_pid) f.push_back({c->d_force_pid, c->sys.size() * kForcePidWords * sizeof(double)});
  if (c->gdir[hcur]) {  // collision histories (GJK warm start)
    f.push_back({c->gdir[hcur], n * c->hist_cap * sizeof(GjkDir)});
    f.push_back({c->gdir_n[hcur], n * sizeof(int)});
  }
  return f;
}

int take_snapshot(grains_gpu_ctx* c, Snapshot& s) {
  s.cur = c->cur;
  s.hcur = c->hcur;
  s.since_gather = c->since_gather;
  s.pending = c->pending_kick2;
  s.pending_dt = c->pending_dt;
  s.steps_done = c->steps_done;
  for (auto& f : snapshot_fields(c, c->cur, c->hcur)) {
    void* q = nullptr;
    if (cudaMalloc(&q, f.second) != cudaSuccess) return GRAINS_GPU_CUDA_ERROR;
    s.bufs.push_back({q, f.second});
    if (cudaMemcpyAsync(q, f.first, f.second, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
      return GRAINS_GPU_CUDA_ERROR;
  }
  return cudaStreamSynchronize(c->stream) == cudaSuccess ? 0 : GRAINS_GPU_CUDA_ERROR;
}

int restore_snapshot(grains_gpu_ctx* c, const Snapshot& s) {
  auto f = snapshot_fields(c, s.cur, s.hcur);
  for (size_t k = 0; k < f.size() && k < s.bufs.size(); ++k)
    if (cudaMemcpyAsync(f[k].first, s.bufs[k].first, f[k].second, cudaMemcpyDeviceToDevice, c->stream) !=
        cudaSuccess)
      return GRAINS_GPU_CUDA_ERROR;
  c->cur = s.cur;
  c->hcur = s.hcur;
  c->since_gather = s.since_gather;
  c->pending_kick2 = s.pending;
  c->pending_dt = s.pending_dt;
  c->steps_done = s.steps_done;
  c->sorted = false;
  c->keys_valid = false;
  if (cudaMemsetAsync(c->stats, 0, sizeof(StatsDev), c->stream) != cudaSuccess) return GRAINS_GPU_CUDA_ERROR;
  return cudaStreamSynchronize(c->stream) == cudaSuccess ? 0 : GRAINS_GPU_CUDA_ERROR;
}

void free_snapshot(Snapshot& s) {
  for (auto& b : s.bufs) cudaFree(b.first);
  s.bufs.clear();
}
}  // namespace

int grains_gpu_autotune(grains_gpu_ctx* c, double time, double dt, int32_t trial_steps, grains_gpu_tuning* best,
                        double* best_ms) {
  if (!c || !best || trial_steps < 1 || !(dt > 0.)) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  if (int rc = flush_kick(c)) return rc;
  Snapshot snap;
  if (take_snapshot(c, snap)) {
    free_snapshot(snap);
    return fail(c, GRAINS_GPU_CUDA_ERROR, "autotune: snapshot failed");
  }
  grains_gpu_tuning cur;
  grains_gpu_get_tuning(c, &cur);
  cur.list_capacity = c->clist_cap;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // time of trial_steps steps from the snapshot (after one untimed run
  // that builds the step graphs); < 0 when the tuning fails (list overflow)
  auto trial = [&](const grains_gpu_tuning& t) -> double {
    if (grains_gpu_set_tuning(c, &t)) return -1.;
    double ms_best = -1.;
    for (int rep = 0; rep < 2; ++rep) {
      if (restore_snapshot(c, snap)) return -1.;
      double tt = time;
      cudaEventRecord(e0, c->stream);
      int rc = grains_gpu_step(c, trial_steps, &tt, dt);
      cudaEventRecord(e1, c->stream);
      if (rc || cudaEventSynchronize(e1) != cudaSuccess) return -1.;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep == 1) ms_best = ms;
    }
    return ms_best;
  };
  double t_best = trial(cur);
  grains_gpu_tuning b = cur;
  // coordinate descent: list capacity, force block, broadphase block, cell factor
  const int caps_sphere[] = {16, 24, 32}, caps_convex[] = {32, 48, 64};
  const int* caps = c->has_convex ? caps_convex : caps_sphere;
  for (int k = 0; k < 3; ++k) {
    grains_gpu_tuning t = b;
    t.list_capacity = caps[k];
    if (t.list_capacity == b.list_capacity) continue;
    const double ms = trial(t);
    if (ms > 0. && (t_best < 0. || ms < t_best)) { t_best = ms; b = t; }
  }
  for (int fb : {64, 128}) {
    grains_gpu_tuning t = b;
    t.forces_block = fb;
    if (fb == b.forces_block) continue;
    const double ms = trial(t);
    if (ms > 0. && (t_best < 0. || ms < t_best)) { t_best = ms; b = t; }
  }
  for (int cb : {128, 256}) {
    grains_gpu_tuning t = b;
    t.contacts_block = cb;
    if (cb == b.contacts_block) continue;
    const double ms = trial(t);
    if (ms > 0. && (t_best < 0. || ms < t_best)) { t_best = ms; b = t; }
  }
  for (int ge : {1, 2, 4, 8, 16}) {
    grains_gpu_tuning t = b;
    t.gather_every = ge;
    if (ge == b.gather_every) continue;
    const double ms = trial(t);
    if (ms > 0. && (t_best < 0. || ms < t_best)) { t_best = ms; b = t; }
  }
  for (int ps : {0, 1}) {
    grains_gpu_tuning t = b;
    t.persistent = ps;
    if (ps == b.persistent) continue;
    const double ms = trial(t);
    if (ms > 0. && (t_best < 0. || ms < t_best)) { t_best = ms; b = t; }
  }
  for (double cf : {1.0, 1.25, 1.5}) {
    grains_gpu_tuning t = b;
    t.cell_factor = cf;
    if (cf == b.cell_factor) continue;
    const double ms = trial(t);
    if (ms > 0. && (t_best < 0. || ms < t_best)) { t_best = ms; b = t; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int rc = grains_gpu_set_tuning(c, &b);
  if (!rc) rc = restore_snapshot(c, snap) ? GRAINS_GPU_CUDA_ERROR : 0;
  free_snapshot(snap);
  if (rc) return fail(c, rc, "autotune: restoring the state failed");
  if (t_best < 0.) return fail(c, GRAINS_GPU_CUDA_ERROR, "autotune: no tuning completed a trial");
  *best = b;
  if (best_ms) *best_ms = t_best;
  return 0;
}

}  // extern "C"

namespace gg {
int launches_per_middle_step() { return 6; }

int context_view(grains_gpu_ctx* c, ContextView* v, std::string& err) {
  if (!c || !v) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) {
    err = "no particles uploaded";
    return GRAINS_GPU_NOT_READY;
  }
  if (int rc = flush_kick(c)) {
    err = c->err;
    return rc;
  }
  const int maxmat = c->cfg.max_materials > 0 ? c->cfg.max_materials : 4;
  *v = ContextView{};
  v->precision = c->precision;
  v->device = c->cfg.device;
  v->stream = c->stream;
  v->n = (int)c->n;
  v->n_cells = c->n_cells;
  v->n_sys = (int)c->sys.size();
  v->n_laws = (int)c->sys.size() * maxmat * maxmat;
  v->hist_cap = c->hist_cap;
  v->spheres_only = c->all_spheres ? 1 : 0;
  v->box_walls_only = 1;
  v->hooke_laws_only = 1;
  for (const auto& s : c->sys) {
    for (const auto& o : s.obs)
      if (c->shapes[o.shape].type != GRAINS_GPU_BOX) v->box_walls_only = 0;
    for (const auto& kv : s.laws)
      if (kv.second.type != GRAINS_GPU_HOOKE && kv.second.type != GRAINS_GPU_HOOKE_MEMORY) v->hooke_laws_only = 0;
  }
  v->n_moving = c->n_moving;
  v->sys = c->d_sys;
  v->shapes = c->d_shapes;
  v->obs = c->d_obs;
  v->cell_obs_start = c->d_cell_obs_start;
  v->cell_obs_idx = c->d_cell_obs_idx;
  v->laws = c->d_laws;
  const auto& b = c->buf[c->cur];
  v->xr = b.xr;
  v->md = b.md;
  v->meta = b.meta;
  v->orig = b.orig;
  v->v = b.v;
  v->w = b.w;
  v->inertia = b.inertia;
  return 0;
}
}  // namespace gg

// ---- reload and RawData files ---------------------------------------------------
namespace {

int io_view(grains_gpu_ctx* c, IoView& v) {
  if (int rc = flush_kick(c)) return rc;
  const auto& b = c->buf[c->cur];
  v = IoView{};
  v.precision = c->precision;
  v.stream = c->stream;
  v.n = (int)c->n;
  v.xr = b.xr;
  v.q = b.q;
  v.basis = c->has_basis ? b.basis : nullptr;
  v.v = b.v;
  v.w = b.w;
  v.F = b.F;
  v.T = b.T;
  v.meta = b.meta;
  v.orig = b.orig;
  v.coord = c->coord;
  v.hist = c->hist[c->hcur];
  v.hist_n = c->hist_n[c->hcur];
  v.hist_cap = c->hist_cap;
  v.row_id = c->d_row_id;
  v.row_sys = c->d_row_sys;
  v.row_keys = c->d_row_keys;
  v.key_rows = c->d_key_rows;
  v.obs_id = c->d_obs_id;
  v.sys_obs_offset = c->d_sys_obs_offset;
  v.attr = c->d_attr;
  v.moved = c->moved;
  return 0;
}

}  // namespace

struct grains_gpu_reload {
  ReloadData d;
  std::string err;
  int status = 0;
};

int grains_gpu_set_record_attributes(grains_gpu_ctx* c, int64_t n, const int32_t* geom_type, const int32_t* tag,
                                     const int32_t* active, const int32_t* transform_type) {
  if (!c || n < 0) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "upload particles first");
  if (n != c->n) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "attributes must cover every uploaded particle");
  std::vector<RecordAttr> a((size_t)n);
  CK(cudaMemcpyAsync(a.data(), c->d_attr, (size_t)n * sizeof(RecordAttr), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int64_t i = 0; i < n; ++i) {
    if (geom_type) a[i].geom_type = geom_type[i];
    if (tag) a[i].tag = tag[i];
    if (active) a[i].active = active[i] ? 1 : 0;
    if (transform_type) a[i].transform_type = transform_type[i];
  }
  CK(cudaMemcpyAsync(c->d_attr, a.data(), (size_t)n * sizeof(RecordAttr), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int grains_gpu_write_reload_particles(grains_gpu_ctx* c, const char* path, int32_t binary, int64_t* bytes) {
  if (!c || !path) return GRAINS_GPU_INVALID_ARGUMENT;
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  IoView v;
  if (int rc = io_view(c, v)) return rc;
  int64_t nb = 0;
  std::string err;
  if (int rc = write_reload_particles(v, c->io, path, binary ? 1 : 0, &nb, err)) return fail(c, rc, err);
  if (bytes) *bytes = nb;
  return 0;
}

int grains_gpu_write_rawdata(grains_gpu_ctx* c, const char* root, double time, int32_t system, int32_t n_total,
                             int32_t binary, int32_t truncate, int64_t* bytes) {
  if (!c || !root || n_total < 0) return GRAINS_GPU_INVALID_ARGUMENT;
  if (system < 0 || system >= (int)c->sys.size()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "bad system index");
  if (!c->uploaded) return fail(c, GRAINS_GPU_NOT_READY, "no particles uploaded");
  IoView v;
  if (int rc = io_view(c, v)) return rc;
  int64_t nb = 0;
  std::string err;
  if (int rc = write_rawdata(v, c->io, root, time, system, n_total, binary ? 1 : 0, truncate ? 1 : 0, &nb, err))
    return fail(c, rc, err);
  if (bytes) *bytes = nb;
  return 0;
}

int grains_gpu_reload_open(const char* path, int32_t binary, grains_gpu_reload** out) {
  if (!path || !out) return GRAINS_GPU_INVALID_ARGUMENT;
  grains_gpu_reload* r = new grains_gpu_reload;
  r->status = read_reload_particles(path, binary ? 1 : 0, r->d, r->err);
  *out = r;  // returned even on failure, so that the message can be read
  return r->status;
}

int grains_gpu_reload_last_error(const grains_gpu_reload* r, char* buf, size_t len) {
  if (!r || !buf || !len) return GRAINS_GPU_INVALID_ARGUMENT;
  std::snprintf(buf, len, "%s", r->err.c_str());
  return 0;
}

int grains_gpu_reload_get(const grains_gpu_reload* r, grains_gpu_reload_data* o) {
  if (!r || !o) return GRAINS_GPU_INVALID_ARGUMENT;
  if (r->status) return r->status;
  const ReloadData& d = r->d;
  const size_t n = d.id.size(), m = d.owner.size();
  o->n_particles = (int64_t)n;
  o->n_memory = (int64_t)m;
  auto put = [](auto* dst, const auto& src) {
    if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
  };
  put(o->geom_type, d.geom_type);
  put(o->id, d.id);
  put(o->tag, d.tag);
  put(o->active, d.active);
  put(o->transform_type, d.transform_type);
  put(o->position, d.position);
  put(o->basis, d.basis);
  put(o->velocity, d.velocity);
  put(o->quaternion, d.quaternion);
  put(o->omega, d.omega);
  put(o->force, d.force);
  put(o->torque, d.torque);
  o->memory.n = (int64_t)m;
  put(o->memory.owner, d.owner);
  put(o->memory.other, d.other);
  put(o->memory.kdelta, d.kdelta);
  put(o->memory.prev_normal, d.prev_normal);
  put(o->memory.spring_torque, d.spring_torque);
  return 0;
}

int grains_gpu_reload_close(grains_gpu_reload* r) {
  delete r;
  return 0;
}

int grains_gpu_format_double(double x, int32_t digits, char* out, size_t cap, int32_t* length) {
  if (!out || digits < 0 || digits > 16) return GRAINS_GPU_INVALID_ARGUMENT;
  const int n = gg::fmt::grains_double_host(x, digits, out, cap);
  if (n < 0) return GRAINS_GPU_INVALID_ARGUMENT;
  if (length) *length = n;
  return 0;
}

int grains_gpu_format_doubles(const double* x, int64_t n, int32_t digits, char* out, int64_t cap, int64_t* length) {
  if ((!x && n) || !out || n < 0 || digits < 0 || digits > 16 || !length) return GRAINS_GPU_INVALID_ARGUMENT;
  std::string err;
  return format_doubles(x, n, digits, out, cap, length, err);
}
