// device_state.h -- layout of the device-resident state of a context and the
// launch interface between the C ABI (api.cu) and the per-precision kernel
// translation units (kernels_fp64.cu, kernels_mixed.cu).
//
// HBM layout (N = particles of all systems, C = cells of all systems):
//   particles are kept sorted by (global cell, id) and re-sorted after every
//   move; two copies of every per-particle array alternate (cur / alt).
//     xr     double4  (x, y, z, circumscribed radius)       32 B
//     q      double4  quaternion (x, y, z, w)                32 B
//     basis  double[9] rotation part of the transform       72 B (non-spheres only)
//     v, w, wbf, F, T  R4 (R = float or double)            16/32 B each
//     inertia R4 (Ixx, Iyy, Izz, 0)
//     md     double4 (mass, crust, equivalent radius, 0)
//     meta   int4    (id, material, shape, system)
//     orig   int     upload index (history row, download order)
//   cells: count[C], start[C+1] (exclusive scan), perm[N] (cell slot ->
//     particle; the identity right after the arrays are gathered in cell order)
//   contact memory: rows of H entries per particle, indexed by upload
//     index, double buffered (prev -> next each force evaluation).
//   contact lists (scratch of a force evaluation): L entries per particle
//     (clist), the result of each entry (res_f, res_t: R4 each) and the work
//     items of the owned entries (work: int4 per entry at most).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/grains_gpu.h"
#include "common.cuh"
#include "contact_law.cuh"

namespace gg {

template <typename R>
struct Vec4;
template <>
struct Vec4<float> {
  using type = float4;
};
template <>
struct Vec4<double> {
  using type = double4;
};

// The collision history of a convex pair (CollisionHistory, Component/src/
// CollisionHistory.cpp:22-49, kept by Particle::InterAction when
// <CollisionDetection History="ON">, Particle.cpp:486-505): the last GJK
// iterate of the pair, as seen from the pair's owner (the lower id) towards
// the partner; other = the partner's id, or kNoGjkDir for an empty slot.
struct GjkDir {
  int other;
  int pad;
  double v[3];
};
constexpr int kNoGjkDir = -2147483647 - 1;

// The narrowphase result of one work item from the GJK kernel (the features of
// RigidBodyWithCrust::ClosestPoint): contact point, overlap vector, overlap
// distance; status 0 features, 1 ContactError even after the crust-x10 retry,
// 2 bounding spheres apart; handled = the retry was used.
struct GjkOut {
  double point[3];
  double ov[3];
  double overlap;
  int status;
  int handled;
};

struct ShapeDev {
  int type;
  int nverts;
  int vert_offset;  // into the vertex table
  int pad;
  double radius;       // sphere / cylinder radius
  double half_height;  // cylinder
  double ext[3];       // box half edges
  double circ;         // circumscribed radius
  double scaling_ext[3];  // local bounding-box half extents (RigidBodyWithCrust scaling)
  double volume;
};

struct SysDev {
  double ox, oy, oz;  // grid origin
  double ex, ey, ez;  // cell edges
  double gx, gy, gz;  // gravity
  int nbi, nbj, nbk;
  int cell_offset;
  int law_offset;
  int n_mat;
  int obs_offset;  // first obstacle of the system in the obstacle table
  int n_obs;
  int moving_offset;  // first entry of the system in the moving-obstacle list
  int n_moving;
  int pad[2];
};

struct ObstacleDev {
  double b[9];   // basis
  double o[3];   // origin
  double bbc[3], bbe[3];  // world AABB centre / half extent
  double vel[3], omega[3];  // current velocity of the centre and angular velocity (zero until the first move)
  int load_first, load_count;  // its imposed motions in the loading table
  int sys;
  double crust;
  double circ;
  double scaling[3];
  int id;
  int material;
  int shape;
  int moving;
  int force_slot;  // its index among the force-driven obstacles, -1 if none
  int moved;       // its imposed velocities moved it in the last move
};

// force-driven obstacles (imposed-force loadings): at most this many per
// context; their contact forces are summed by kForceBlocks blocks, each
// writing partial sums that the obstacle move adds up in block order
constexpr int kMaxForceObstacles = 4;
constexpr int kForceBlocks = 148;
// the imposed-force controller's history per system: the previous two force
// differences and the previous displacement, then the flag of a non-zero
// contact force met
constexpr int kForcePidWords = 10;

// One imposed motion of an obstacle (ObstacleImposedVelocity), directions
// normalised and phases in radians as its XML constructor leaves them
// (ObstacleImposedVelocity.cpp:60-262).  An imposed force
// (GRAINS_GPU_FORCE_TRANSLATION, ObstacleImposedForce.cpp:29-80) keeps its
// force in vel, its direction in unit, its mass in amp (<= 0: automatic) and
// Vmax in period.
struct LoadingDev {
  int type, has_center;
  double ts, te;
  double vel[3], unit[3], omega[3], center[3];
  double amp, period, phase;
  double mamp[3], mper[3], mphase[3];
};

template <typename R>
struct HistEntry {
  int other;  // neighbour id (particle) or obstacle table index (flags & 1)
  int flags;
  R kd[3];
  R n[3];
  R sp[3];
};

struct StatsDev {
  unsigned long long n_cand;
  unsigned long long n_obs_cand;
  unsigned long long n_contacts;
  unsigned long long n_obs_contacts;
  unsigned long long n_gjk_calls;
  unsigned long long n_gjk_iters;
  unsigned long long overlap_max_bits;
  double overlap_sum;
  int status;
  int pad;
};

template <typename R>
struct ParticleArrays {
  double4* xr;
  double4* q;
  double* basis;
  typename Vec4<R>::type* v;
  typename Vec4<R>::type* w;
  typename Vec4<R>::type* wbf;
  typename Vec4<R>::type* F;
  typename Vec4<R>::type* T;
  typename Vec4<R>::type* inertia;
  double4* md;
  int4* meta;
  int* orig;
  unsigned* key;  // cell key of the current positions (written by the kick / bin kernels)
};

template <typename R>
struct StepArgs {
  int n;                 // particles
  int n_cells;           // total cells
  int n_sys;
  int hist_cap;          // H
  int has_basis;         // non-spherical particles present
  int has_convex;        // a pair may need GJK (non-sphere particle or non-box obstacle)
  const SysDev* sys;
  const ShapeDev* shapes;
  const double* verts;   // polyhedron vertices (xyz)
  const int* adj_start;  // polyhedron vertex adjacency: per vertex (vertex table index) its first
  const int* adj;        // neighbour in adj (local vertex indices); adj_start has one entry more
  const ObstacleDev* obs;
  const int* cell_obs_start;  // static obstacle CSR per cell (C+1)
  const int* cell_obs_idx;
  const int* moving_idx;
  const LoadingDev* loads;    // imposed obstacle motions
  int* load_flags;            // per system: a loading active over this step, over the previous one
  const LawParams<R>* laws;
  ParticleArrays<R> cur;
  ParticleArrays<R> alt;
  int* coord;            // coordination number (sorted order)
  int* cell_count;
  int* cell_cursor;      // fill cursor of each cell (scatter)
  int* cell_start;
  int* block_sums;
  int* perm;
  HistEntry<R>* hist_prev;
  int* hist_n_prev;
  HistEntry<R>* hist_next;
  int* hist_n_next;
  StatsDev* stats;
  int* clist;            // per-particle contact lists, clist_cap entries each: a contacting
                         // particle's slot (| 1 << 30 when this particle owns the pair) or
                         // -1 - obstacle index for a candidate obstacle
  int* ccount;
  int clist_cap;
  typename Vec4<R>::type* res_f;  // per list entry: force on this particle, w = contact flag
  typename Vec4<R>::type* res_t;  // per list entry: torque on this particle
  int4* work;            // owned list entries of this evaluation: (particle, entry, index | memory rank << 9,
                         // memory row)
  int* work_n;           // their count (cleared by the sums kernel)
  int* pairs;            // diagnostic contact pair output (2 ints per pair) or null
  int pairs_cap;
  unsigned long long* pairs_n;
  double* pair_force;    // diagnostic: force on the lower id of each contact pair (3 doubles) or null
  int* pair_sys;         // diagnostic: system of each contact pair
  double gjk_tol;
  int fluid_corrected;   // immersed particles: accelerations divided by 1 - rho_f / rho_p (md.w = rho_f / rho_p)
  const double* hydro;   // per upload index: the fluid's force and torque (6 doubles), or null
  int gjk_sv;            // the signed-volume GJK for non-spherical pairs
  int gjk_accel;         // Nesterov-accelerated GJK directions (<CollisionDetection Acceleration="ON">)
  int gjk_history;       // warm-started GJK from the pair's collision history (History="ON")
  GjkOut* gjk_out;       // per work item: the GJK kernel's narrowphase result (null: GJK inline in the pair kernel)
  int* gjk_next;         // the GJK kernel's work-item counter (cleared by the sums kernel)
  int* gjk_order;        // the GJK work items grouped by shape pair (work-item capacity)
  int* gjk_bins;         // per shape-pair bin: counts, then placement cursors (2 x 32 ints)
  GjkDir* gdir_prev;     // collision histories of the last evaluation (rows of hist_cap slots by memory row)
  int* gdir_n_prev;
  GjkDir* gdir_next;     // written by this evaluation
  int* gdir_n_next;
  long long barrier_polls;  // persistent kernel: polls before a grid-barrier wait gives up
  int barrier_skip_block;   // persistent kernel: a block that leaves at once (a test of the bounded wait), or -1
  int contacts_block;    // threads per block of contacts_kernel (<= 256)
  int forces_block;      // threads per block of forces_kernel (<= 128)
};

// kernel launchers, instantiated for float and double
template <typename R>
int launch_kick_move(const StepArgs<R>& a, cudaStream_t s, int do_kick2, double dt_kick2, int do_move,
                     double dt_v, double dt_x);
template <typename R>
int launch_bin(const StepArgs<R>& a, cudaStream_t s);
// cell ranges and the slot -> particle permutation of the current positions;
// gather != 0 also permutes the particle arrays into cell order (into the
// other buffer; the permutation becomes the identity)
template <typename R>
int launch_sort_and_gather(const StepArgs<R>& a, cudaStream_t s, int gather, int gather_forces);
// phases (bits): 1 = contact lists, 2 = pair narrowphase and law, 4 = per-particle sums
template <typename R>
// kick != 0: the sums kernel also applies the second half kick and the next
// step's first half kick, drift and binning (a middle step)
int launch_forces(const StepArgs<R>& a, cudaStream_t s, double dt, int diag, int phases = 7, int kick = 0);
template <typename R>
int launch_zero_kdelta(const StepArgs<R>& a, cudaStream_t s);
// device arrays in upload order of grains_gpu_update_particles (basis may be null)
struct KinematicStage {
  const double *position, *quaternion, *velocity, *omega, *basis;
};
// device arrays in upload order of grains_gpu_download_particles (any may be null)
struct DownloadStage {
  double *position, *quaternion, *basis, *velocity, *omega, *force, *torque;
  int *coordination, *id;
};
template <typename R>
int launch_update_dynamic(const StepArgs<R>& a, cudaStream_t s, const KinematicStage& st);
// velocities and angular velocities (world, upload order) of every particle
template <typename R>
int launch_set_velocities(const StepArgs<R>& a, cudaStream_t s, const double* vel, const double* omega);
// md.w = rho_f / rho_p of every particle from ratio (upload order)
template <typename R>
int launch_set_fluid_ratio(const StepArgs<R>& a, cudaStream_t s, const double* ratio);
// the kinematic state of the upload indices rows[0 .. n_rows) from stage
// entries 0 .. n_rows (slot_of: n ints of scratch)
template <typename R>
int launch_update_rows(const StepArgs<R>& a, cudaStream_t s, const KinematicStage& st, const long long* rows,
                       long long n_rows, int* slot_of);
template <typename R>
int launch_pack_download(const StepArgs<R>& a, cudaStream_t s, const DownloadStage& d);
template <typename R>
int launch_candidate_pairs(const StepArgs<R>& a, cudaStream_t s, int sys, int include_obstacles, int* out,
                           int cap, unsigned long long* count);
// moves every moving obstacle over dt (defined in kernels_mixed.cu)
// force_part / force_pid: the force-driven obstacles' partial contact forces
// and the systems' controller histories (nullptr: no force-driven obstacle)
int launch_obstacle_move(ObstacleDev* obs, const int* moving_idx, int n_moving, const LoadingDev* loads,
                         int* load_flags, int n_sys, const ShapeDev* shapes, const double* verts, double dt,
                         double* clock, double host_time, int use_host_time, const double* force_part,
                         double* force_pid, cudaStream_t s);
// the contact forces on the force-driven obstacles: kForceBlocks partial sums
// per obstacle into force_part (fixed assignment and order)
template <typename R>
int launch_obstacle_force(const StepArgs<R>& a, double* force_part, int n_obs, cudaStream_t s);
// n middle steps of grains_gpu_step in one cooperative launch of `blocks`
// blocks (persistent_blocks: all resident); bar: 2 zeroed unsigned of grid
// barrier state, sums: `blocks` ints of scan scratch
template <typename R>
int persistent_blocks(const StepArgs<R>& a);
template <typename R>
int launch_persistent_steps(const StepArgs<R>& a, cudaStream_t s, int n_steps, double dt, int gather_every,
                            int since_gather, int n_moving, double* clock, unsigned* bar, int* sums, int blocks);
// number of kernel launches issued by one middle step of grains_gpu_step
int launches_per_middle_step();

}  // namespace gg
