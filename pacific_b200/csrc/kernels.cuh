// kernels.cuh -- sm_100a kernels of the Grains3D DEM time step, templated on
// the arithmetic type R of velocities, forces, the contact law and the
// contact memory (float: mixed precision, double: plain FP64).  Positions,
// quaternions, bases and every contact decision are double in both.
//
// One DEM step (KDK leapfrog, Grains.cpp:344-364) is:
//   kick_move      second half kick of the previous step (when pending),
//                  first half kick + drift + rotation (SecondOrderLeapFrog),
//                  new cell key and per-cell count (fire-and-forget atomic)
//   scan x2        exclusive scan of the per-cell counts -> cell ranges
//   scatter        slot = atomic fill cursor of the cell
//   cell_sort      each cell's particles ordered by id (deterministic order)
//   gather         every per-particle array permuted into the new order
//                  (every few steps only: between gathers the kernels reach
//                  a cell's particles through the permutation)
//   forces         broadphase over the 27 surrounding cells, sphere/box
//                  narrowphase, contact law + memory, per-particle sums,
//                  static and moving obstacles
// The second half kick of the last step is flushed by kick_move with
// do_move = 0.
#pragma once

#include <algorithm>

#include <cooperative_groups.h>

#include "common.cuh"
#include "contact_law.cuh"
#include "device_state.h"
#include "sphere_contact.cuh"
#include "gjk.cuh"

namespace gg {

namespace cg = cooperative_groups;

template <typename R>
using R4 = typename Vec4<R>::type;

template <typename R>
__device__ __forceinline__ V3<R> ld3(const R4<R>& a) {
  return v3<R>(a.x, a.y, a.z);
}
template <typename R>
__device__ __forceinline__ R4<R> st3(V3<R> a, R wv = R(0)) {
  R4<R> r;
  r.x = a.x;
  r.y = a.y;
  r.z = a.z;
  r.w = wv;
  return r;
}

__device__ __forceinline__ void set_status(StatsDev* st, int bits) { atomicOr(&st->status, bits); }

// Cell::GetCell (Base/src/Cell.cpp:172-184) + LinkedCell::getCell validity
__device__ __forceinline__ bool cell_of(const SysDev& S, double x, double y, double z, int& i, int& j, int& k) {
  i = int(floor(xdiv(xsub(x, S.ox), S.ex)));
  j = int(floor(xdiv(xsub(y, S.oy), S.ey)));
  k = int(floor(xdiv(xsub(z, S.oz), S.ez)));
  bool ok = -1 < i && i < S.nbi && -1 < j && j < S.nbj && -1 < k && k < S.nbk;
  if (!ok) {
    i = min(max(i, 0), S.nbi - 1);
    j = min(max(j, 0), S.nbj - 1);
    k = min(max(k, 0), S.nbk - 1);
  }
  return ok;
}
// LinkedCell::getCellNumber (LinkedCell.cpp:1165-1168) + system offset
__device__ __forceinline__ int cell_index(const SysDev& S, int i, int j, int k) {
  return S.cell_offset + j * S.nbk * S.nbi + k * S.nbi + i;
}

// ---------------------------------------------------------------------------
// Angular acceleration in the body frame (ParticleKinematicsSphere.cpp:47-54,
// ParticleKinematics3D.cpp:56-75 with predictor mode on, Grains.cpp:18)
template <typename R>
__device__ __forceinline__ V3<R> dwdt(bool sphere, V3<R> I, V3<R> Tbf, V3<R> om, R cf) {
  if (sphere) return v3<R>(Tbf.x / (cf * I.x), Tbf.y / (cf * I.y), Tbf.z / (cf * I.z));
  return v3<R>(Tbf.x / (cf * I.x) + om.y * om.z * (I.y - I.z) / I.x,
               Tbf.y / (cf * I.y) + om.z * om.x * (I.z - I.x) / I.y,
               Tbf.z / (cf * I.z) + om.x * om.y * (I.x - I.y) / I.z);
}
// SSP-RK3 of SecondOrderLeapFrog::Move / advanceVelocity (SecondOrderLeapFrog.cpp:55-68)
template <typename R>
__device__ __forceinline__ V3<R> rk3(bool sphere, V3<R> I, V3<R> Tbf, V3<R> wbf, R dt, R cf) {
  V3<R> K1 = sc(dwdt(sphere, I, Tbf, wbf, cf), dt);
  V3<R> K2 = sc(dwdt(sphere, I, Tbf, wbf + K1, cf), dt);
  V3<R> K3 = sc(dwdt(sphere, I, Tbf, wbf + sc(K1 + K2, R(0.25)), cf), dt);
  return wbf + dv((K1 + K2) + sc(K3, R(4)), R(6));
}

// ---------------------------------------------------------------------------
// integrate: optional pending second half kick (SecondOrderLeapFrog::
// advanceVelocity, SecondOrderLeapFrog.cpp:74-95), then ParticleKinematics::
// Move (ParticleKinematics.cpp:62-105) and the cell key of the new position.
// Reads particle s of `src`, writes it to slot s of `dst` (dst == src: in
// place).  F and T are the torsor of the last force evaluation.
template <typename R>
__device__ __forceinline__ void integrate(const StepArgs<R>& a, const ParticleArrays<R>& src,
                                          const ParticleArrays<R>& dst, int s, V3<R> F, V3<R> T, int do_kick2,
                                          R dt_kick2, int do_move, R dt_v, double dt_x) {
  double4 xr = src.xr[s];
  const double4 qd = src.q[s];
  const int4 meta = src.meta[s];
  const double4 md = src.md[s];
  V3<R> v = ld3<R>(src.v[s]), w = ld3<R>(src.w[s]), wbf = ld3<R>(src.wbf[s]);
  const V3<R> I = ld3<R>(src.inertia[s]);
  const bool sphere = a.shapes[meta.z].type == 0;
  const R mass = R(md.x);
  // the coupling factor of an immersed particle (ParticleKinematics::
  // setCouplingFactor, ParticleKinematics.cpp:483-488): 1 - rho_f / rho_p when
  // the acceleration is corrected, else 1 (md.w = rho_f / rho_p, 0 in air)
  const R cf = a.fluid_corrected ? R(1. - md.w) : R(1);
  Qt<double> q{v3<double>(qd.x, qd.y, qd.z), qd.w};
  const Qt<R> qr{v3<R>(R(qd.x), R(qd.y), R(qd.z)), R(qd.w)};
  if (do_kick2) {
    V3<R> Tbf = q_to_body(qr, T);
    v = v + sc(dv(F, mass * cf), dt_kick2);
    wbf = rk3(sphere, I, Tbf, wbf, dt_kick2, cf);
    w = q_to_world(qr, wbf);
  }
  if (do_move) {
    V3<R> Tbf = q_to_body(qr, T);
    v = v + sc(dv(F, mass * cf), dt_v);
    V3<double> tm = sc(v3<double>(double(v.x), double(v.y), double(v.z)), dt_x);
    wbf = rk3(sphere, I, Tbf, wbf, dt_v, cf);
    w = q_to_world(qr, wbf);
    V3<R> meanw = w;
    xr.x = xr.x + tm.x;
    xr.y = xr.y + tm.y;
    xr.z = xr.z + tm.z;
    V3<double> mw = v3<double>(double(meanw.x), double(meanw.y), double(meanw.z));
    double nom = norm(mw);
    Qt<double> dq{v3<double>(0., 0., 0.), 1.};
    if (nom > kEpsilon) {
      double c = cos(nom * dt_x / 2.), sn = sin(nom * dt_x / 2.);
      dq = Qt<double>{sc(mw, sn * 1. / nom), c};
    }
    q = qmul(dq, q);
    if (a.has_basis) {
      M3 b;
      for (int t = 0; t < 9; ++t) b.m[t] = src.basis[9 * (size_t)s + t];
      mrotate_left(b, dq);
      for (int t = 0; t < 9; ++t) dst.basis[9 * (size_t)s + t] = b.m[t];
    }
    if (norm(tm) > md.y) set_status(a.stats, GRAINS_GPU_MOTION_ERROR);
    // new cell key, counted in its cell
    const SysDev& S = a.sys[meta.w];
    int ci, cj, ck;
    if (!cell_of(S, xr.x, xr.y, xr.z, ci, cj, ck)) set_status(a.stats, GRAINS_GPU_OUT_OF_GRID);
    unsigned key = (unsigned)cell_index(S, ci, cj, ck);
    dst.key[s] = key;
    atomicAdd(&a.cell_count[key], 1);  // result unused: a fire-and-forget reduction
  } else if (a.has_basis && dst.basis != src.basis) {
    for (int t = 0; t < 9; ++t) dst.basis[9 * (size_t)s + t] = src.basis[9 * (size_t)s + t];
  }
  dst.xr[s] = xr;
  dst.q[s] = make_double4(q.v.x, q.v.y, q.v.z, q.w);
  dst.v[s] = st3<R>(v);
  dst.w[s] = st3<R>(w);
  dst.wbf[s] = st3<R>(wbf);
}

// kick_move: integrate in place (the per-phase entry points and the first step
// of a run)
template <typename R>
__global__ void __launch_bounds__(256) kick_move_kernel(StepArgs<R> a, int do_kick2, R dt_kick2, int do_move,
                                                        R dt_v, double dt_x) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  integrate(a, a.cur, a.cur, s, ld3<R>(a.cur.F[s]), ld3<R>(a.cur.T[s]), do_kick2, dt_kick2, do_move, dt_v, dt_x);
}

// bin: cell keys of the current positions (after an upload)
template <typename R>
__global__ void bin_kernel(StepArgs<R> a) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  double4 xr = a.cur.xr[s];
  int4 meta = a.cur.meta[s];
  const SysDev& S = a.sys[meta.w];
  int ci, cj, ck;
  if (!cell_of(S, xr.x, xr.y, xr.z, ci, cj, ck)) set_status(a.stats, GRAINS_GPU_OUT_OF_GRID);
  unsigned key = (unsigned)cell_index(S, ci, cj, ck);
  a.cur.key[s] = key;
  atomicAdd(&a.cell_count[key], 1);
}

// ---------------------------------------------------------------------------
// exclusive scan of cell counts: 1024 threads x 4 items per block
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
  __shared__ int warp_sums[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int ws = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += y;
    }
    if (lane < nw) warp_sums[lane] = ws;
  }
  __syncthreads();
  int base = wid > 0 ? warp_sums[wid - 1] : 0;
  *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

// The launched sort of a step scans the cell counts within tiles of kScanTile
// cells only: each tile's local exclusive prefix (into the cursor array), its
// total, and the counts zeroed.  The scatter then counts every cell's
// particles again, taking each particle's rank in its cell from that atomic,
// and adds the start of its tile (the sum of the totals before it); the cell
// sort writes the final cell starts.  No second pass over the cells.
static __global__ void __launch_bounds__(kScanThreads) scan_tiles_kernel(int* counts, int* local_start, int* tile_sums,
                                                                         int n) {
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int vals[kScanItems];
  int sum = 0;
#pragma unroll
  for (int t = 0; t < kScanItems; ++t) {
    vals[t] = (base + t < n) ? counts[base + t] : 0;
    sum += vals[t];
  }
  int total;
  int pre = block_exclusive_scan(sum, &total);
#pragma unroll
  for (int t = 0; t < kScanItems; ++t) {
    if (base + t < n) {
      local_start[base + t] = pre;
      counts[base + t] = 0;
    }
    pre += vals[t];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// the start of every tile (exclusive prefix of the tile totals) in shared
// memory; every thread of the block calls it
constexpr int kMaxScanTiles = 4096;
__device__ __forceinline__ void tile_starts(const int* tile_sums, int n_tiles, int* start) {
  const int per = (n_tiles + blockDim.x - 1) / blockDim.x;
  const int t0 = threadIdx.x * per;
  int sum = 0;
  for (int k = 0; k < per; ++k)
    if (t0 + k < n_tiles) sum += tile_sums[t0 + k];
  int total;
  int pre = block_exclusive_scan(sum, &total);
  for (int k = 0; k < per; ++k)
    if (t0 + k < n_tiles) {
      start[t0 + k] = pre;
      pre += tile_sums[t0 + k];
    }
  __syncthreads();
}

// slot of each particle in its cell's range; the order inside a cell is
// fixed afterwards by cell_sort_kernel (by id), so the atomic order does not
// matter
template <typename R>
__device__ __forceinline__ void scatter_one(const StepArgs<R>& a, int s) {
  const unsigned key = a.cur.key[s];
  const long long slot = (key < (unsigned)a.n_cells) ? (long long)atomicAdd(&a.cell_cursor[key], 1) : -1;
  if (slot < 0 || slot >= a.n) {
    set_status(a.stats, GRAINS_GPU_CUDA_ERROR);
    return;
  }
  a.perm[slot] = s;
}

// the launched scatter: slot = start of the key's tile + the cell's start in
// the tile + the particle's rank from the cell's count
template <typename R>
__global__ void __launch_bounds__(256) scatter_kernel(StepArgs<R> a) {
  __shared__ int tile_start[kMaxScanTiles];
  tile_starts(a.block_sums, (a.n_cells + kScanTile - 1) / kScanTile, tile_start);
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const unsigned key = a.cur.key[s];
  const long long slot =
      (key < (unsigned)a.n_cells)
          ? (long long)tile_start[key / kScanTile] + a.cell_cursor[key] + atomicAdd(&a.cell_count[key], 1)
          : -1;
  if (slot < 0 || slot >= a.n) {
    set_status(a.stats, GRAINS_GPU_CUDA_ERROR);
    return;
  }
  a.perm[slot] = s;
}

// order the slots [b, e) of cell c by particle id; resets the count for the
// next step
template <typename R>
__device__ __forceinline__ void cell_sort_range(const StepArgs<R>& a, int c, int b, int e) {
  a.cell_count[c] = 0;
  if (b < 0 || e > a.n || b > e) return;
  for (int i = b + 1; i < e; ++i) {
    int pi = a.perm[i];
    int idi = a.cur.meta[pi].x;
    int j = i - 1;
    while (j >= b && a.cur.meta[a.perm[j]].x > idi) {
      a.perm[j + 1] = a.perm[j];
      --j;
    }
    a.perm[j + 1] = pi;
  }
}

// the cell sort of a fully scanned cell list (the persistent kernel's)
template <typename R>
__device__ __forceinline__ void cell_sort_one(const StepArgs<R>& a, int c) {
  cell_sort_range(a, c, a.cell_start[c], a.cell_start[c + 1]);
}

// the launched cell sort: the final start of each cell (its tile's start + its
// start in the tile; its end from the count the scatter rebuilt), then the
// sort.  The block's 256 cells lie in one tile; the block sums the totals of
// the tiles before it.
constexpr int kCellSortThreads = 256;
static_assert(kScanTile % kCellSortThreads == 0, "a cell-sort block must lie in one scan tile");
template <typename R>
__global__ void __launch_bounds__(kCellSortThreads) cell_sort_kernel(StepArgs<R> a) {
  __shared__ int warp_part[kCellSortThreads / 32];
  const int c = blockIdx.x * kCellSortThreads + threadIdx.x;
  const int tile = (blockIdx.x * kCellSortThreads) / kScanTile;
  int part = 0;
  for (int t = threadIdx.x; t < tile; t += kCellSortThreads) part += a.block_sums[t];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = part;
  __syncthreads();
  int start = 0;
#pragma unroll
  for (int w = 0; w < kCellSortThreads / 32; ++w) start += warp_part[w];
  if (c < a.n_cells) {
    const int b = start + a.cell_cursor[c], e = b + a.cell_count[c];
    a.cell_start[c] = b;
    if (c == a.n_cells - 1) a.cell_start[c + 1] = e;
    cell_sort_range(a, c, b, e);
  }
}

// permutes every per-particle array into cell order; the permutation then
// becomes the identity (each thread resets its own entry after reading it)
template <typename R>
__device__ __forceinline__ void gather_one(const StepArgs<R>& a, int t, int gather_forces) {
  int s = a.perm[t];
  if (s < 0 || s >= a.n) {
    set_status(a.stats, GRAINS_GPU_CUDA_ERROR);
    return;
  }
  a.perm[t] = t;
  const ParticleArrays<R>& C = a.cur;
  const ParticleArrays<R>& D = a.alt;
  D.xr[t] = C.xr[s];
  D.q[t] = C.q[s];
  D.v[t] = C.v[s];
  D.w[t] = C.w[s];
  D.wbf[t] = C.wbf[s];
  D.inertia[t] = C.inertia[s];
  D.md[t] = C.md[s];
  D.meta[t] = C.meta[s];
  D.orig[t] = C.orig[s];
  D.key[t] = C.key[s];
  if (gather_forces) {
    D.F[t] = C.F[s];
    D.T[t] = C.T[s];
  }
  if (a.has_basis) {
    for (int k = 0; k < 9; ++k) D.basis[9 * (size_t)t + k] = C.basis[9 * (size_t)s + k];
  }
}

template <typename R>
__global__ void __launch_bounds__(256) gather_kernel(StepArgs<R> a, int gather_forces) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < a.n) gather_one(a, t, gather_forces);
}

// ---------------------------------------------------------------------------
// Contact memory lookup in the owner's row of the previous step, in two
// parts so that the loads of the row start with the pair's other loads: the
// entry count and the keys of the first 4 entries (MemoryKeys), then the match
// and the payload of the matched entry; longer rows continue one entry at a
// time.
struct MemoryKeys {
  int n;
  int2 key[4];
};

template <typename R>
__device__ __forceinline__ MemoryKeys memory_keys(const StepArgs<R>& a, int row) {
  const HistEntry<R>* h = a.hist_prev + (size_t)row * a.hist_cap;
  MemoryKeys k;
  k.n = a.hist_n_prev[row];
#pragma unroll
  for (int j = 0; j < 4; ++j) k.key[j] = j < a.hist_cap ? make_int2(h[j].other, h[j].flags) : make_int2(-1, -1);
  return k;
}

template <typename R>
__device__ __forceinline__ bool find_memory(const StepArgs<R>& a, int row, const MemoryKeys& k, int other, int flags,
                                            PairMemory<R>& m) {
  const HistEntry<R>* h = a.hist_prev + (size_t)row * a.hist_cap;
  int found = -1;
#pragma unroll
  for (int j = 3; j >= 0; --j)
    if (j < k.n && k.key[j].x == other && k.key[j].y == flags) found = j;
  for (int j = 4; found < 0 && j < k.n; ++j)
    if (h[j].other == other && h[j].flags == flags) found = j;
  if (found < 0) return false;
  const HistEntry<R>& e = h[found];
  m.kdelta = v3<R>(e.kd[0], e.kd[1], e.kd[2]);
  m.prev_normal = v3<R>(e.n[0], e.n[1], e.n[2]);
  m.spring = v3<R>(e.sp[0], e.sp[1], e.sp[2]);
  return true;
}

template <typename R>
__device__ __forceinline__ void store_memory(const StepArgs<R>& a, int row, int& cnt, int other, int flags,
                                             const PairMemory<R>& m) {
  if (cnt >= a.hist_cap) {
    set_status(a.stats, GRAINS_GPU_HISTORY_FULL);
    return;
  }
  HistEntry<R> e;
  e.other = other;
  e.flags = flags;
  e.kd[0] = m.kdelta.x; e.kd[1] = m.kdelta.y; e.kd[2] = m.kdelta.z;
  e.n[0] = m.prev_normal.x; e.n[1] = m.prev_normal.y; e.n[2] = m.prev_normal.z;
  e.sp[0] = m.spring.x; e.sp[1] = m.spring.y; e.sp[2] = m.spring.z;
  a.hist_next[(size_t)row * a.hist_cap + cnt] = e;
  ++cnt;
}

__device__ __forceinline__ void atomic_max_pos_double(unsigned long long* addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// Applies the contact law for the pair (p0, p1) seen from p0 and returns the
// force on p0, its rolling torque, and the torques of the contact force about
// both centres (lever0 x f, lever1 x (-f); Torsor::addForce, Torsor.cpp:184-189).
// The mixed path (R = float) forms the normal part of the law in double from
// `pd` (normal_part_fp64), and takes the normal force's share of the torques in
// double: for spheres the lever is parallel to the normal, so lever x f_normal
// vanishes, but the FP32 product of the two rounded vectors leaves a residue of
// 1e-7 |lever| |f|, which can exceed the true torque of the tangential force.
// The FP64 path runs the reference's expressions throughout.
template <typename R>
__device__ __forceinline__ LawResult<R> pair_law(const LawParams<R>& L, R dt, const ContactGeom& g,
                                                 const BodyAtContact<R>& b0, const BodyAtContact<R>& b1,
                                                 const PairFp64& pd, bool existed, PairMemory<R>& mem, V3<R>& t0,
                                                 V3<R>& t1) {
  if constexpr (sizeof(R) == 4) {
    const V3<double> pen = v3<double>(g.overlap_vector.x, g.overlap_vector.y, g.overlap_vector.z);
    const NormalFp64<R> nd = normal_part_fp64(L, pen, -g.overlap, pd);
    const V3<double> tn0 = cross(pd.lev0, nd.delFN64), tn1 = cross(pd.lev1, -nd.delFN64);
    const LawResult<R> res = apply_contact_law_fp64_normal(L, dt, nd, b0, b1, existed, mem);
    t0 = v3<R>(R(tn0.x), R(tn0.y), R(tn0.z)) + cross(b0.lever, res.tangential);
    t1 = v3<R>(R(tn1.x), R(tn1.y), R(tn1.z)) + cross(b1.lever, -res.tangential);
    return res;
  } else {
    const LawResult<R> res =
        apply_contact_law(L, dt, from_d3<R>(g.overlap_vector), R(-g.overlap), b0, b1, existed, mem);
    t0 = cross(b0.lever, res.force);
    t1 = cross(b1.lever, -res.force);
    return res;
  }
}

template <typename R>
__device__ __forceinline__ V3<double> widen(V3<R> a) {
  return v3<double>(double(a.x), double(a.y), double(a.z));
}
__device__ __forceinline__ V3<double> dvec(D3 a) { return v3<double>(a.x, a.y, a.z); }

// Contact with a pair error: RigidBodyWithCrust::ClosestPoint_ErreurHandling
// (RigidBodyWithCrust.cpp:532-588) for two spheres, whose crust-x10 shrunk
// bodies are spheres of radius r * max((r - 10 crust) / r, 0.5): the contact
// is imposed with an overlap equal to minus the crust sum along B->A.
__device__ __forceinline__ ContactGeom sphere_sphere_error_handling(D3 A, double ra, double ca, D3 B, double rb,
                                                                    double cb, bool& fatal) {
  double sa = fmax(xdiv(xsub(ra, xmul(10., ca)), ra), 0.5);
  double sb = fmax(xdiv(xsub(rb, xmul(10., cb)), rb), 0.5);
  D3 ab = xsub3(B, A);
  double nab = xnorm(ab);
  double ras = xmul(ra, sa), rbs = xmul(rb, sb);
  double dist = xsub(nab, xadd(ras, rbs));
  ContactGeom g;
  fatal = dist < kEpsilon;
  D3 u = xdivs(ab, nab);
  D3 pa = xadd3(A, xscale(u, ras));
  D3 pb = xsub3(B, xscale(u, rbs));
  g.point = xadd3(xdivs(pa, 2.0), xdivs(pb, 2.0));
  double imp = xmul(1., xadd(ca, cb));
  g.overlap_vector = xscale(d3(-u.x, -u.y, -u.z), imp);
  g.overlap = -imp;
  g.status = 0;
  return g;
}


// ---------------------------------------------------------------------------
// general convex narrowphase glue
template <typename R>
__device__ __forceinline__ void make_body_ref(const StepArgs<R>& a, int shape, int slot, double crust, BodyRef& b) {
  const ShapeDev& sh = a.shapes[shape];
  const double4 xr = a.cur.xr[slot];
  b.type = sh.type;
  b.nverts = sh.nverts;
  b.verts = a.verts + 3 * sh.vert_offset;
  b.radius = xr.w;
  b.cyl_r = sh.radius;
  b.cyl_hh = sh.half_height;
  b.ext = d3(sh.ext[0], sh.ext[1], sh.ext[2]);
  b.crust = crust;
  if (a.has_basis) {
    for (int t = 0; t < 9; ++t) b.basis.m[t] = a.cur.basis[9 * (size_t)slot + t];
  } else {
    for (int t = 0; t < 9; ++t) b.basis.m[t] = (t % 4 == 0) ? 1. : 0.;
  }
  b.origin = d3(xr.x, xr.y, xr.z);
  b.adj_start = sh.type == GRAINS_GPU_POLYHEDRON ? a.adj_start + sh.vert_offset : nullptr;
  b.adj = a.adj;
  for (int i = 0; i < 3; ++i) b.lext[i] = sh.type == GRAINS_GPU_SPHERE ? xr.w : sh.scaling_ext[i];
  for (int i = 0; i < 3; ++i) b.scaling[i] = b.lext[i] < kEpsilon ? 1. : xdiv(xsub(b.lext[i], crust), b.lext[i]);
}

template <typename R>
__device__ __forceinline__ void make_obstacle_ref(const StepArgs<R>& a, int oidx, BodyRef& b) {
  const ObstacleDev& O = a.obs[oidx];
  const ShapeDev& sh = a.shapes[O.shape];
  b.type = sh.type;
  b.nverts = sh.nverts;
  b.verts = a.verts + 3 * sh.vert_offset;
  b.radius = O.circ;
  b.cyl_r = sh.radius;
  b.cyl_hh = sh.half_height;
  b.ext = d3(sh.ext[0], sh.ext[1], sh.ext[2]);
  b.crust = O.crust;
  for (int t = 0; t < 9; ++t) b.basis.m[t] = O.b[t];
  b.origin = d3(O.o[0], O.o[1], O.o[2]);
  b.adj_start = sh.type == GRAINS_GPU_POLYHEDRON ? a.adj_start + sh.vert_offset : nullptr;
  b.adj = a.adj;
  for (int i = 0; i < 3; ++i) b.scaling[i] = O.scaling[i];
  for (int i = 0; i < 3; ++i) b.lext[i] = sh.scaling_ext[i];
}

// Closest point of a general pair: the double GJK in both precisions (the
// mixed path keeps FP32 for the contact law only).  An FP32 GJK is not used:
// on curved bodies it often stops in Johnson's backup procedure with distance
// errors up to 2e-5 m, far above typical overlaps, and even as a separation
// filter (certified by its support-plane lower bound) it made the drum's
// force kernel 3x slower than the double GJK alone on B200 (0.67 vs 0.22 ms
// per step, 100,000 convex bodies).  Error handling (crust x10) on
// ContactError.  st carries the accelerated-direction option and, for a
// warm-started run, the pair's direction in and out.
template <typename R, bool SV = false>
__device__ ContactGeom convex_closest_point(const StepArgs<R>& a, const BodyRef& A, const BodyRef& B, int& iters,
                                            int& handled, GjkStart<double>& st) {
  handled = 0;
  ContactGeom c = SV ? convex_closest_point_sv(A, B, a.gjk_tol, &iters, &st)
                     : convex_closest_point_t<double>(A, B, a.gjk_tol, &iters, nullptr, nullptr, &st);
  if (c.status == 1) {
    c = convex_error_handling(A, B, A.lext, B.lext, 10., a.gjk_tol, st.accel);
    handled = 1;
  }
  return c;
}

// The collision history of an owned pair in the owner's row of the last
// evaluation (CollisionHistory::lookupCollision, CollisionHistory.cpp:41-49).
// The reference also looks the pair up, negated, in the partner's map
// (Particle.cpp:491-495); here a pair's history always lives with its owner,
// the lower id, so that second place is never needed.
template <typename R>
__device__ __forceinline__ bool find_gjk_dir(const StepArgs<R>& a, int row, int other, V3<double>& v) {
  const int n = a.gdir_n_prev[row];
  const GjkDir* g = a.gdir_prev + (size_t)row * a.hist_cap;
  for (int k = 0; k < n; ++k)
    if (g[k].other == other) {
      v = v3<double>(g[k].v[0], g[k].v[1], g[k].v[2]);
      return true;
    }
  return false;
}

// ---------------------------------------------------------------------------
// The force evaluation runs in three phases.
//
// A. contacts (one thread per particle, cell-sorted order): the broadphase over
//    the 27 surrounding cells with the exact double overlap test, then the
//    obstacles linked to the particle's cell.  Each particle gets a list of
//    entries: a contacting particle's slot, with kOwnBit set when this particle
//    owns the pair (the lower id), or -1 - k for a candidate obstacle k.  Every
//    owned entry (owned pairs and obstacles) becomes a work item.
// B. pairs (one thread per work item): the narrowphase, the contact memory of
//    the owner and the contact law, ONCE per pair.  The owner writes the
//    results of both sides: its own entry's slot gets (f, lever_p0 x f + M) and
//    the partner's entry for the pair (found in the partner's list) gets (-f,
//    lever_p1 x (-f) - M), the exact values the partner would compute with the
//    law from its side; and the updated memory goes to the owner's row at the
//    entry's rank among its owned entries.
// C. sums (one thread per particle): weight + every entry's result in list
//    order (deterministic: no float atomics), coordination, and the owner's
//    memory row packed (entries without a contact or without a memory law
//    leave a hole that is squeezed out here).

constexpr int kOwnBit = 1 << 30;  // list entry: this particle owns the pair
__device__ __forceinline__ int entry_slot(int e) { return e & (kOwnBit - 1); }
__device__ __forceinline__ bool entry_owned(int e) { return e < 0 || (e & kOwnBit); }

// contacts: the broadphase and the exact bounding-sphere test.  For every
// neighbour j != i of the 27 surrounding cells (LinkedCell::ComputeForces as a
// set, LinkedCell.cpp:1019-1103) it tests |x_j - x_i| - (r_i + r_j) < 0 in
// double with the reference's rounding (for spheres this is the contact
// decision of ClosestPointSPHERESPHERE, RigidBodyWithCrust.cpp:611-613; for
// other convex bodies the circumscribed-sphere prefilter of ClosestPoint,
// :279-282) and appends j's slot.  Then the obstacles of the cell
// (SimpleObstacle::InterAction's candidates, SimpleObstacle.cpp:222-270):
// static ones linked at set-up, moving ones whose box meets the twice-expanded
// cell (LinkedCell.cpp:1568-1585), each kept when its box meets the particle's
// circumscribed sphere box (BBox::InZone).
template <typename R>
__device__ __forceinline__ void contacts_one(const StepArgs<R>& a, int s, unsigned long long& ncand,
                                             unsigned long long& nobs_cand, int& n_work) {
  const ParticleArrays<R>& P = a.cur;
  const double4 xi = P.xr[s];
  const int idi = P.meta[s].x;
  const SysDev& S = a.sys[P.meta[s].w];
  const D3 Xi = d3(xi.x, xi.y, xi.z);
  // the particle's cell from the key of the current positions (the cell lists
  // were built from it): key = offset + j nbk nbi + k nbi + i
  const int local = (int)P.key[s] - S.cell_offset;
  const int ci = local % S.nbi, ck = (local / S.nbi) % S.nbk, cj = local / (S.nbi * S.nbk);
  const int i0 = max(ci - 1, 0), i1 = min(ci + 1, S.nbi - 1);
  // the slot ranges of the 9 cell rows, loaded before any candidate
  int r0[9], r1[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    const int j = cj + r / 3 - 1, k = ck + r % 3 - 1;
    const bool ok = j >= 0 && j < S.nbj && k >= 0 && k < S.nbk;
    r0[r] = ok ? a.cell_start[cell_index(S, i0, j, k)] : 0;
    r1[r] = ok ? a.cell_start[cell_index(S, i1, j, k) + 1] : 0;
  }
  int* list = a.clist + (size_t)s * a.clist_cap;
  int cnt = 0, owned = 0;
  auto test = [&](int p, const double4& xj) {
    // cheap rejection of far candidates: the squared distance against the
    // squared radius sum with a 1e-12 relative margin (rounding of either
    // side is below 1e-15 relative)
    const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const double rs = xi.w + xj.w;
    if (dx * dx + dy * dy + dz * dz > rs * rs * (1. + 1.e-12)) return;
    D3 ab;
    double nab;
    // |AB| and r_A + r_B are symmetric in IEEE arithmetic, so the test
    // gives the same bits whichever body is A: both particles list the pair
    const double dist = sphere_sphere_overlap(Xi, xi.w, d3(xj.x, xj.y, xj.z), xj.w, &ab, &nab);
    if (dist < 0. && p != s) {
      const bool own = idi < P.meta[p].x;
      if (cnt < a.clist_cap) list[cnt] = p | (own ? kOwnBit : 0);
      ++cnt;
      owned += own ? 1 : 0;
    }
  };
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    ncand += (unsigned long long)(r1[r] - r0[r]);
    // two candidates per iteration: their permutation and position loads are
    // in flight together (the list order stays the slot order)
    int t = r0[r];
    for (; t + 1 < r1[r]; t += 2) {
      const int pa = a.perm[t], pb = a.perm[t + 1];  // cell slot -> particle
      const double4 xa = P.xr[pa], xb = P.xr[pb];
      test(pa, xa);
      test(pb, xb);
    }
    if (t < r1[r]) {
      const int pa = a.perm[t];
      test(pa, P.xr[pa]);
    }
  }
  // obstacles linked to the particle's cell
  {
    const int cell = cell_index(S, ci, cj, ck);
    const int ob0 = a.cell_obs_start[cell], ob1 = a.cell_obs_start[cell + 1];
    const int nstat = ob1 - ob0;
    const int ntot = nstat + S.n_moving;
    const D3 cg = d3(xadd(xadd(S.ox, xmul(double(ci), S.ex)), xdiv(S.ex, 2.)),
                     xadd(xadd(S.oy, xmul(double(cj), S.ey)), xdiv(S.ey, 2.)),
                     xadd(xadd(S.oz, xmul(double(ck), S.ez)), xdiv(S.ez, 2.)));
    for (int u = 0; u < ntot; ++u) {
      int oidx;
      if (u < nstat) {
        oidx = a.cell_obs_idx[ob0 + u];
      } else {
        oidx = a.moving_idx[S.moving_offset + (u - nstat)];
        const ObstacleDev& O = a.obs[oidx];
        if (!in_zone(d3(O.bbc[0], O.bbc[1], O.bbc[2]), d3(O.bbe[0], O.bbe[1], O.bbe[2]), cg, S.ex, S.ey, S.ez))
          continue;
      }
      const ObstacleDev& O = a.obs[oidx];
      if (!in_zone(d3(O.bbc[0], O.bbc[1], O.bbc[2]), d3(O.bbe[0], O.bbe[1], O.bbe[2]), Xi, xi.w, xi.w, xi.w))
        continue;
      ++nobs_cand;
      if (cnt < a.clist_cap) list[cnt] = -1 - oidx;
      ++cnt;
      ++owned;
    }
  }
  if (cnt > a.clist_cap) {
    set_status(a.stats, GRAINS_GPU_PAIR_OVERFLOW);
    cnt = a.clist_cap;
  }
  a.ccount[s] = cnt;
  ncand -= 1;  // the particle itself
  n_work = owned;  // recounted by the caller when the list overflowed
}

// work items of the owned entries of particle s, at `base` onward: (particle,
// the entry itself, entry index | memory rank << 9, the particle's memory
// row).  The rank of an owned entry among the particle's owned entries is its
// contact-memory position.  Carrying the entry and the row lets the pair
// kernel issue every load of its second level at once.
template <typename R>
__device__ __forceinline__ void emit_work(const StepArgs<R>& a, int s, int base) {
  const int* list = a.clist + (size_t)s * a.clist_cap;
  const int cnt = a.ccount[s];
  const int row = a.cur.orig[s];
  const long long limit = (long long)a.n * a.clist_cap;  // the work array's size
  int rank = 0;
  for (int q = 0; q < cnt; ++q) {
    const int e = list[q];
    if (!entry_owned(e)) continue;
    if ((long long)base + rank >= limit) {  // a counter left over from an unfinished evaluation
      set_status(a.stats, GRAINS_GPU_CUDA_ERROR);
      return;
    }
    a.work[base + rank] = make_int4(s, e, q | (rank << 9), row);
    ++rank;
  }
}

// warp sum of a per-thread count into a statistics counter (every lane of the
// warp calls it)
__device__ __forceinline__ void warp_add(unsigned long long* dst, unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// one warp-aggregated reservation of work-item slots for every lane's count
// (every lane of the warp calls it); returns the lane's first slot
__device__ __forceinline__ int warp_reserve(int* counter, int count) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int incl = count;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += y;
  }
  const int total = __shfl_sync(full, incl, 31);
  int base = 0;
  if (lane == 31 && total > 0) base = atomicAdd(counter, total);
  base = __shfl_sync(full, base, 31);
  return base + incl - count;
}

// contacts of particles first, first + stride, ... (all particles when the
// threads of the grid start at 0 .. stride - 1); the trip count is uniform
// across a warp for the warp-wide reservation and reductions
template <typename R>
__device__ __forceinline__ void contacts_range(const StepArgs<R>& a, int first, int stride) {
  const int padded = (a.n + stride - 1) / stride * stride;
  unsigned long long ncand = 0, nobs = 0;
  for (int s = first; s < padded; s += stride) {
    int nw = 0;
    if (s < a.n) {
      contacts_one(a, s, ncand, nobs, nw);
      if (nw > 0 && a.ccount[s] == a.clist_cap) {  // the list may have overflowed: count what it holds
        const int* list = a.clist + (size_t)s * a.clist_cap;
        nw = 0;
        for (int q = 0; q < a.clist_cap; ++q) nw += entry_owned(list[q]) ? 1 : 0;
      }
    }
    const int base = warp_reserve(a.work_n, nw);
    if (nw > 0) emit_work(a, s, base);
  }
  warp_add(&a.stats->n_cand, ncand);
  warp_add(&a.stats->n_obs_cand, nobs);
}

// four blocks of 256 per SM (64 registers, a few spills): the candidate loop
// is latency bound, and the fourth block's warps hide more of it (settled 200k
// bed: 0.093 -> 0.078 ms per launch)
#ifndef GG_CONTACTS_MIN_BLOCKS
#define GG_CONTACTS_MIN_BLOCKS 4
#endif
template <typename R>
__global__ void __launch_bounds__(256, GG_CONTACTS_MIN_BLOCKS) contacts_kernel(StepArgs<R> a) {
  contacts_range(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ---------------------------------------------------------------------------
// statistics of the force evaluation, summed per thread then per warp
struct ForceStats {
  unsigned long long ncont_own, nobs_cont, ngjk, ngjk_it;
  double ov_sum, ov_max;
};

__device__ __forceinline__ void flush_force_stats(StatsDev* st, ForceStats& f) {
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    f.ncont_own += __shfl_down_sync(full, f.ncont_own, o);
    f.nobs_cont += __shfl_down_sync(full, f.nobs_cont, o);
    f.ngjk += __shfl_down_sync(full, f.ngjk, o);
    f.ngjk_it += __shfl_down_sync(full, f.ngjk_it, o);
    f.ov_sum += __shfl_down_sync(full, f.ov_sum, o);
    f.ov_max = fmax(f.ov_max, __shfl_down_sync(full, f.ov_max, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (f.ncont_own) atomicAdd(&st->n_contacts, f.ncont_own);
    if (f.nobs_cont) atomicAdd(&st->n_obs_contacts, f.nobs_cont);
    if (f.ngjk) atomicAdd(&st->n_gjk_calls, f.ngjk);
    if (f.ngjk_it) atomicAdd(&st->n_gjk_iters, f.ngjk_it);
    if (f.ov_sum > 0.) atomicAdd(&st->overlap_sum, f.ov_sum);
    if (f.ov_max > 0.) atomic_max_pos_double(&st->overlap_max_bits, f.ov_max);
  }
}

// result of one list entry: (force, flag) and torque; flag 0 = no contact,
// 1 = contact, 3 = contact whose owner stored a memory entry
template <typename R>
__device__ __forceinline__ void put_result(const StepArgs<R>& a, size_t slot, V3<R> f, V3<R> t, int flag) {
  a.res_f[slot] = st3<R>(f, R(flag));
  a.res_t[slot] = st3<R>(t);
}
template <typename R>
__device__ __forceinline__ void put_no_contact(const StepArgs<R>& a, size_t slot) {
  R4<R> z;
  z.x = z.y = z.z = z.w = R(0);
  a.res_f[slot] = z;
}
template <typename R>
__device__ __forceinline__ void put_memory(const StepArgs<R>& a, int row, int rank, int other, int flags,
                                           const PairMemory<R>& m) {
  if (rank >= a.hist_cap) {
    set_status(a.stats, GRAINS_GPU_HISTORY_FULL);
    return;
  }
  HistEntry<R> e;
  e.other = other;
  e.flags = flags;
  e.kd[0] = m.kdelta.x; e.kd[1] = m.kdelta.y; e.kd[2] = m.kdelta.z;
  e.n[0] = m.prev_normal.x; e.n[1] = m.prev_normal.y; e.n[2] = m.prev_normal.z;
  e.sp[0] = m.spring.x; e.sp[1] = m.spring.y; e.sp[2] = m.spring.z;
  a.hist_next[(size_t)row * a.hist_cap + rank] = e;
}

// B. one owned list entry: particle pair (p0 = this particle, the lower id)
// or particle-obstacle candidate (p0 = the particle, p1 = the obstacle)
// GEOM: the narrowphase of general convex pairs comes from the GJK kernel
// (gjk_out) instead of running here
template <typename R, bool DIAG, bool CONVEX, bool SV = false, bool GEOM = false>
__device__ __forceinline__ void pair_one(const StepArgs<R>& a, int idx, int4 item, R dt, ForceStats& fs) {
  const ParticleArrays<R>& P = a.cur;
  const int s = item.x, e = item.y, q = item.z & 511, rank = item.z >> 9, oi = item.w;
  const size_t my_slot = (size_t)s * a.clist_cap + q;
  const double4 xi = P.xr[s];
  const int4 mi = P.meta[s];
  const double4 mdi = P.md[s];
  const V3<R> vi = ld3<R>(P.v[s]);
  const V3<R> wi = ld3<R>(P.w[s]);
  const MemoryKeys keys = memory_keys(a, oi);
  const SysDev& S = a.sys[mi.w];
  const D3 Xi = d3(xi.x, xi.y, xi.z);

  if (e >= 0) {
    // ---- particle pair: this particle (s) is p0, the partner (t) p1
    const int t = entry_slot(e);
    const double4 xj = P.xr[t];
    const int4 mj = P.meta[t];
    // the partner's entry for this pair: its first 16 entries are loaded
    // together (no load waits on a comparison), longer lists continue singly
    const int* tl = a.clist + (size_t)t * a.clist_cap;
    const int tn = a.ccount[t];
    int qp = -1;
    {
      int4 ch[4];
#pragma unroll
      for (int c = 0; c < 4; ++c)
        ch[c] = 4 * c < tn ? reinterpret_cast<const int4*>(tl)[c] : make_int4(-1, -1, -1, -1);
#pragma unroll
      for (int c = 3; c >= 0; --c) {
        const int v[4] = {ch[c].w, ch[c].z, ch[c].y, ch[c].x};
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (v[u] == s && 4 * c + 3 - u < tn) qp = 4 * c + 3 - u;  // a partner's entry for s never has kOwnBit
      }
      for (int k = 16; qp < 0 && k < tn; ++k)
        if (tl[k] == s) qp = k;
    }
    const size_t other_slot = (size_t)t * a.clist_cap + (qp < 0 ? 0 : qp);
    const D3 Xj = d3(xj.x, xj.y, xj.z);
    ContactGeom g;
    bool contact = true;
    const double4 mdj = P.md[t];
    if (!CONVEX || (a.shapes[mi.z].type == GRAINS_GPU_SPHERE && a.shapes[mj.z].type == GRAINS_GPU_SPHERE)) {
      D3 ab;
      double nab;
      const double dist = sphere_sphere_overlap(Xi, xi.w, Xj, xj.w, &ab, &nab);
      contact = dist < 0.;
      if (contact) {
        g = sphere_sphere_features(Xi, xi.w, ab, nab, dist, xadd(mdi.y, mdj.y));
        if (g.status) {
          bool fatal;
          g = sphere_sphere_error_handling(Xi, xi.w, mdi.y, Xj, xj.w, mdj.y, fatal);
          set_status(a.stats, fatal ? GRAINS_GPU_CONTACT_ERROR : GRAINS_GPU_CONTACT_HANDLED);
          contact = !fatal;
        }
      }
    } else if constexpr (GEOM) {
      // the GJK kernel's result for this work item
      g = gjk_result(a.gjk_out[idx]);
      contact = g.status == 0 && g.overlap < 0.;
    } else {
      // general convex pair: circumscribed-sphere test then GJK on crust-shrunk bodies
      BodyRef ba, bb;
      make_body_ref(a, mi.z, s, mdi.y, ba);
      make_body_ref(a, mj.z, t, mdj.y, bb);
      int it = 0, handled = 0;
      GjkStart<double> st;
      st.accel = a.gjk_accel != 0;
      st.history = a.gjk_history != 0;
      bool known = false;
      if (st.history) known = find_gjk_dir(a, oi, mj.x, st.v0);
      const V3<double> v_before = st.v0;
      g = convex_closest_point<R, SV>(a, ba, bb, it, handled, st);
      if (g.status != 2) {
        ++fs.ngjk;
        fs.ngjk_it += it;
      }
      if (handled) set_status(a.stats, g.status == 1 ? GRAINS_GPU_CONTACT_ERROR : GRAINS_GPU_CONTACT_HANDLED);
      contact = g.status == 0 && g.overlap < 0.;
      if (st.history && rank < a.hist_cap) {
        // CollisionHistory::updateCollision / removeCollision (Particle.cpp:
        // 497-501): the run's last iterate is kept, apart bounding spheres
        // remove the entry, and a ContactError leaves it as it was
        GjkDir d;
        d.other = mj.x;
        d.pad = 0;
        const V3<double> keep = handled ? v_before : st.v0;
        if ((handled && !known) || (keep.x == 0. && keep.y == 0. && keep.z == 0.)) d.other = kNoGjkDir;
        d.v[0] = keep.x;
        d.v[1] = keep.y;
        d.v[2] = keep.z;
        a.gdir_next[(size_t)oi * a.hist_cap + rank] = d;
      }
    }
    if (CONVEX && a.gjk_history && rank < a.hist_cap &&
        (a.shapes[mi.z].type == GRAINS_GPU_SPHERE && a.shapes[mj.z].type == GRAINS_GPU_SPHERE))
      a.gdir_next[(size_t)oi * a.hist_cap + rank].other = kNoGjkDir;
    if (!contact) {
      put_no_contact(a, my_slot);
      if (qp >= 0) put_no_contact(a, other_slot);
      return;
    }
    if (qp < 0) set_status(a.stats, GRAINS_GPU_PAIR_OVERFLOW);  // the partner's list overflowed
    const V3<R> vj = ld3<R>(P.v[t]), wj = ld3<R>(P.w[t]);
    const D3 lev0 = xsub3(g.point, Xi), lev1 = xsub3(g.point, Xj);
    BodyAtContact<R> b0, b1;
    b0.v = vi;
    b0.w = wi;
    b0.lever = from_d3<R>(lev0);
    b0.pos_minus_contact = from_d3<R>(xsub3(Xi, g.point));
    b0.mass = R(mdi.x);
    b0.req = R(mdi.z);
    b1.v = vj;
    b1.w = wj;
    b1.lever = from_d3<R>(lev1);
    b1.pos_minus_contact = from_d3<R>(xsub3(Xj, g.point));
    b1.mass = R(mdj.x);
    b1.req = R(mdj.z);
    const LawParams<R> L = a.laws[S.law_offset + mi.y * S.n_mat + mj.y];
    PairMemory<R> mem;
    bool existed = false;
    if (law_has_memory(L.type)) existed = find_memory(a, oi, keys, mj.x, 0, mem);
    PairFp64 pd;
    if constexpr (sizeof(R) == 4) {
      pd.v0 = widen(vi);
      pd.w0 = widen(wi);
      pd.lev0 = dvec(lev0);
      pd.v1 = widen(vj);
      pd.w1 = widen(wj);
      pd.lev1 = dvec(lev1);
      pd.m0 = mdi.x;
      pd.m1 = mdj.x;
      pd.req0 = mdi.z;
      pd.req1 = mdj.z;
    }
    V3<R> t0, t1;
    LawResult<R> res = pair_law(L, dt, g, b0, b1, pd, existed, mem, t0, t1);
    int flag = 1;
    if (law_has_memory(L.type)) {
      put_memory(a, oi, rank, mj.x, 0, mem);
      flag = 3;
    }
    // p0 gets f at the contact point, p1 gets -f (and the rolling torques +M / -M)
    if (law_has_torque(L)) {
      t0 = t0 + res.torque;
      t1 = t1 + (-res.torque);
    }
    put_result(a, my_slot, res.force, t0, flag);
    if (qp >= 0) put_result(a, other_slot, -res.force, t1, 1);
    ++fs.ncont_own;
    const double o = fabs(g.overlap);
    fs.ov_sum += o;
    fs.ov_max = fmax(fs.ov_max, o);
    if (DIAG && a.pairs) {
      unsigned long long slot = atomicAdd(a.pairs_n, 1ull);
      if (slot < (unsigned long long)a.pairs_cap) {
        a.pairs[2 * slot] = mi.x;
        a.pairs[2 * slot + 1] = mj.x;
        a.pair_sys[slot] = mi.w;
        if (a.pair_force) {
          a.pair_force[3 * slot] = double(res.force.x);
          a.pair_force[3 * slot + 1] = double(res.force.y);
          a.pair_force[3 * slot + 2] = double(res.force.z);
        }
      }
    }
    return;
  }

  // ---- obstacle candidate (SimpleObstacle::InterAction, SimpleObstacle.cpp:222-270)
  if (CONVEX && a.gjk_history && rank < a.hist_cap) a.gdir_next[(size_t)oi * a.hist_cap + rank].other = kNoGjkDir;
  const int oidx = -1 - e;
  const ObstacleDev& O = a.obs[oidx];
  const D3 oo = d3(O.o[0], O.o[1], O.o[2]);
  const ShapeDev& sho = a.shapes[O.shape];
  ContactGeom g;
  if (!CONVEX || (a.shapes[mi.z].type == GRAINS_GPU_SPHERE && sho.type == GRAINS_GPU_BOX)) {
    M3 ob;
    for (int k = 0; k < 9; ++k) ob.m[k] = O.b[k];
    g = sphere_box(Xi, xi.w, xadd(mdi.y, O.crust), ob, oo, d3(sho.ext[0], sho.ext[1], sho.ext[2]));
    if (g.status) {
      set_status(a.stats, GRAINS_GPU_CONTACT_ERROR);
      g.overlap = 1.;
    }
  } else if constexpr (GEOM) {
    g = gjk_result(a.gjk_out[idx]);
    if (g.status != 0) g.overlap = 1.;
  } else {
    BodyRef ba, bb;
    make_body_ref(a, mi.z, s, mdi.y, ba);
    make_obstacle_ref(a, oidx, bb);
    int it = 0, handled = 0;
    GjkStart<double> st;  // no collision history for obstacles (SimpleObstacle.cpp:222-250)
    st.accel = a.gjk_accel != 0;
    g = convex_closest_point<R, SV>(a, ba, bb, it, handled, st);
    if (g.status != 2) {
      ++fs.ngjk;
      fs.ngjk_it += it;
    }
    if (handled) set_status(a.stats, g.status == 1 ? GRAINS_GPU_CONTACT_ERROR : GRAINS_GPU_CONTACT_HANDLED);
    if (g.status != 0) g.overlap = 1.;
  }
  if (!(g.overlap < 0.)) {
    put_no_contact(a, my_slot);
    return;
  }
  // p0 = particle, p1 = obstacle (mass 1e20, velocity at the point, Obstacle.cpp:128-133)
  BodyAtContact<R> b0, b1;
  b0.v = vi;
  b0.w = wi;
  b0.lever = from_d3<R>(xsub3(g.point, Xi));
  b0.pos_minus_contact = from_d3<R>(xsub3(Xi, g.point));
  b0.mass = R(mdi.x);
  b0.req = R(mdi.z);
  // the law adds w x lever to the centre velocity (velocity_at)
  const D3 olev = xsub3(g.point, oo);
  b1.v = v3<R>(R(O.vel[0]), R(O.vel[1]), R(O.vel[2]));
  b1.w = v3<R>(R(O.omega[0]), R(O.omega[1]), R(O.omega[2]));
  b1.lever = from_d3<R>(olev);
  b1.pos_minus_contact = from_d3<R>(xsub3(oo, g.point));
  b1.mass = R(kObstacleMass);
  b1.req = R(pow((0.75 / kPi) * sho.volume, 1. / 3.));
  const LawParams<R> L = a.laws[S.law_offset + mi.y * S.n_mat + O.material];
  PairMemory<R> mem;
  const int oloc = oidx - S.obs_offset;
  bool existed = false;
  if (law_has_memory(L.type)) existed = find_memory(a, oi, keys, oloc, 1, mem);
  PairFp64 pd;
  if constexpr (sizeof(R) == 4) {
    pd.v0 = widen(vi);
    pd.w0 = widen(wi);
    pd.lev0 = dvec(xsub3(g.point, Xi));
    pd.v1 = v3<double>(O.vel[0], O.vel[1], O.vel[2]);
    pd.w1 = v3<double>(O.omega[0], O.omega[1], O.omega[2]);
    pd.lev1 = dvec(olev);
    pd.m0 = mdi.x;
    pd.m1 = kObstacleMass;
    pd.req0 = mdi.z;
    pd.req1 = pow((0.75 / kPi) * sho.volume, 1. / 3.);
  }
  V3<R> t0, t1;
  LawResult<R> res = pair_law(L, dt, g, b0, b1, pd, existed, mem, t0, t1);
  int flag = 1;
  if (law_has_memory(L.type)) {
    put_memory(a, oi, rank, oloc, 1, mem);
    flag = 3;
  }
  if (law_has_torque(L)) t0 = t0 + res.torque;
  put_result(a, my_slot, res.force, t0, flag);
  ++fs.nobs_cont;
  const double o = fabs(g.overlap);
  fs.ov_sum += o;
  fs.ov_max = fmax(fs.ov_max, o);
}

// ---------------------------------------------------------------------------
// B0. The GJK phase of convex scenarios (Johnson's GJK): every work item whose
// pair needs the general narrowphase gets RigidBodyWithCrust::ClosestPoint's
// features written to gjk_out[item]; the pair kernel then applies the law.
//
// The runs take 1 to 30+ iterations, so one run per thread leaves most lanes
// of a warp idle while the longest run of the warp finishes (5 of 32 lanes
// active on the settled drum).  Here each thread keeps a run in flight and
// takes the next work item as soon as its run ends: every pass of the loop is
// one GJK iteration on every busy lane.  The arithmetic of a run is that of
// gjk_distance (same state, same passes), so results do not depend on the
// schedule.

__device__ __forceinline__ ContactGeom gjk_result(const GjkOut& o) {
  ContactGeom g;
  g.point = d3(o.point[0], o.point[1], o.point[2]);
  g.overlap_vector = d3(o.ov[0], o.ov[1], o.ov[2]);
  g.overlap = o.overlap;
  g.status = o.status;
  return g;
}

// whether a work item's pair needs the general narrowphase (the sphere-sphere
// and sphere-box cases of ClosestPoint are analytic, RigidBodyWithCrust.cpp:
// 218-258)
template <typename R>
__device__ __forceinline__ bool needs_gjk(const StepArgs<R>& a, int4 item) {
  const int ts = a.shapes[a.cur.meta[item.x].z].type;
  if (item.y >= 0) return !(ts == GRAINS_GPU_SPHERE && a.shapes[a.cur.meta[entry_slot(item.y)].z].type == GRAINS_GPU_SPHERE);
  return !(ts == GRAINS_GPU_SPHERE && a.shapes[a.obs[-1 - item.y].shape].type == GRAINS_GPU_BOX);
}

// the bodies of a work item: p0 = the particle, p1 = the partner or obstacle
template <typename R>
__device__ __forceinline__ void item_bodies(const StepArgs<R>& a, int4 item, BodyRef& ba, BodyRef& bb) {
  const int s = item.x;
  make_body_ref(a, a.cur.meta[s].z, s, a.cur.md[s].y, ba);
  if (item.y >= 0) {
    const int t = entry_slot(item.y);
    make_body_ref(a, a.cur.meta[t].z, t, a.cur.md[t].y, bb);
  } else {
    make_obstacle_ref(a, -1 - item.y, bb);
  }
}

// one work-item index per calling lane, from a warp-aggregated atomic
__device__ __forceinline__ int take_item(int* counter) {
  cg::coalesced_group g = cg::coalesced_threads();
  int base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(counter, (int)g.size());
  return g.shfl(base, 0) + (int)g.thread_rank();
}

template <typename R>
struct GjkLane {
  int idx;        // work item in flight
  int4 item;
  double crust_sum;
  bool known;     // the pair's history was found
  V3<double> v_before;
  LocalBody<double> la, lb;
  GjkRun<double> run;
};

// the collision history of a particle pair (Particle.cpp:497-504): the run's
// last iterate, or the entry as it was when a ContactError was handled, or a
// hole (bounding spheres apart, zero direction)
template <typename R>
__device__ __forceinline__ void store_gjk_dir(const StepArgs<R>& a, int4 item, int partner_id, int status,
                                              int handled, bool known, V3<double> before, V3<double> after) {
  const int rank = item.z >> 9;
  if (rank >= a.hist_cap) return;
  GjkDir d;
  d.other = partner_id;
  d.pad = 0;
  const V3<double> keep = handled ? before : after;
  if (status == 2 || (handled && !known) || (keep.x == 0. && keep.y == 0. && keep.z == 0.)) d.other = kNoGjkDir;
  d.v[0] = keep.x;
  d.v[1] = keep.y;
  d.v[2] = keep.z;
  a.gdir_next[(size_t)item.w * a.hist_cap + rank] = d;
}

// takes work items until one needs a GJK run and starts it; items whose
// bounding spheres are apart are finished on the way.  False when none is left.
template <typename R>
__device__ bool gjk_lane_start(const StepArgs<R>& a, int n_gjk, GjkLane<R>& L) {
  for (;;) {
    const int j = take_item(a.gjk_next);
    if (j >= n_gjk) return false;
    const int k = a.gjk_order[j];  // the GJK items grouped by shape pair
    const int4 item = a.work[k];
    BodyRef ba, bb;
    item_bodies(a, item, ba, bb);
    const bool pair = item.y >= 0;
    const int partner = pair ? a.cur.meta[entry_slot(item.y)].x : 0;
    GjkStart<double> st;
    st.accel = a.gjk_accel != 0;
    st.history = pair && a.gjk_history != 0;
    L.known = st.history && find_gjk_dir(a, item.w, partner, st.v0);
    const D3 g = xsub3(ba.origin, bb.origin);
    if (!(xnorm(g) < xadd(ba.radius, bb.radius))) {  // RigidBodyWithCrust.cpp:278-282
      GjkOut& o = a.gjk_out[k];
      o.status = 2;
      o.handled = 0;
      o.overlap = 1.;
      if (st.history) store_gjk_dir(a, item, partner, 2, 0, L.known, st.v0, st.v0);
      continue;
    }
    L.idx = k;
    L.item = item;
    L.crust_sum = xadd(ba.crust, bb.crust);
    L.v_before = st.v0;
    L.la = local_body<double>(ba, d3(0., 0., 0.), ba.scaling);
    L.lb = local_body<double>(bb, d3(0., 0., 0.), bb.scaling);
    gjk_begin(L.run, L.la, L.lb, a.gjk_tol, st);  // L.run.g: the lane's shared-memory arrays
    return true;
  }
}

// the features of a finished run, the crust-x10 retry on ContactError, the
// history and the statistics
template <typename R>
__device__ void gjk_lane_finish(const StepArgs<R>& a, GjkLane<R>& L, unsigned long long& ngjk,
                                unsigned long long& nit) {
  const GjkResult<double> r = gjk_end(L.run, L.la, L.lb);
  ContactGeom c = gjk_features(r, L.crust_sum, d3(0., 0., 0.));
  ++ngjk;
  nit += r.iters;
  int handled = 0;
  if (c.status == 1) {
    BodyRef ba, bb;
    item_bodies(a, L.item, ba, bb);
    c = convex_error_handling(ba, bb, ba.lext, bb.lext, 10., a.gjk_tol, a.gjk_accel != 0);
    handled = 1;
    set_status(a.stats, c.status == 1 ? GRAINS_GPU_CONTACT_ERROR : GRAINS_GPU_CONTACT_HANDLED);
  }
  GjkOut& o = a.gjk_out[L.idx];
  o.point[0] = c.point.x;
  o.point[1] = c.point.y;
  o.point[2] = c.point.z;
  o.ov[0] = c.overlap_vector.x;
  o.ov[1] = c.overlap_vector.y;
  o.ov[2] = c.overlap_vector.z;
  o.overlap = c.overlap;
  o.status = c.status;
  o.handled = handled;
  if (L.item.y >= 0 && a.gjk_history)
    store_gjk_dir(a, L.item, a.cur.meta[entry_slot(L.item.y)].x, c.status, handled, L.known, L.v_before, r.v);
}

// The GJK items are grouped by the shape types of their pair first (a
// counting sort into kGjkBins bins), so that the lanes of a warp run the same
// support functions: counts per bin, then each item placed in its bin.
constexpr int kGjkBins = 32;
template <typename R>
__device__ __forceinline__ int gjk_bin(const StepArgs<R>& a, int4 item) {
  const int ta = a.shapes[a.cur.meta[item.x].z].type;
  const int tb = item.y >= 0 ? a.shapes[a.cur.meta[entry_slot(item.y)].z].type
                             : 4 + a.shapes[a.obs[-1 - item.y].shape].type;
  return ta * 8 + tb;
}

template <typename R>
__global__ void __launch_bounds__(256) gjk_count_kernel(StepArgs<R> a) {
  __shared__ int h[kGjkBins];
  if (threadIdx.x < kGjkBins) h[threadIdx.x] = 0;
  __syncthreads();
  const int n_items = (int)min((long long)*(volatile int*)a.work_n, (long long)a.n * a.clist_cap);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_items; k += gridDim.x * blockDim.x) {
    const int4 item = a.work[k];
    if (needs_gjk(a, item)) atomicAdd(&h[gjk_bin(a, item)], 1);
  }
  __syncthreads();
  if (threadIdx.x < kGjkBins && h[threadIdx.x]) atomicAdd(&a.gjk_bins[threadIdx.x], h[threadIdx.x]);
}

// Each block places a contiguous range of work items, a tile at a time: the
// tile's bin counts in shared memory, one global reservation per bin and tile,
// then each warp's items of a bin placed by one shared-memory atomic (the
// lanes' ranks from __match_any_sync).  One global atomic per item on the 32
// bin cursors took 169 us per step on the settled drum (550,000 items).
constexpr int kPlaceTile = 2048;
template <typename R>
__global__ void __launch_bounds__(256) gjk_place_kernel(StepArgs<R> a) {
  __shared__ int base[kGjkBins], count[kGjkBins], cursor[kGjkBins];
  __shared__ signed char tile_bin[kPlaceTile];
  if (threadIdx.x == 0) {
    int sum = 0;
    for (int b = 0; b < kGjkBins; ++b) {
      base[b] = sum;
      sum += a.gjk_bins[b];
    }
  }
  const unsigned full = 0xffffffffu;
  const unsigned lt = (1u << (threadIdx.x & 31)) - 1u;  // lanes below this one
  const int n_items = (int)min((long long)*(volatile int*)a.work_n, (long long)a.n * a.clist_cap);
  const int chunk = (n_items + gridDim.x - 1) / gridDim.x;
  const int lo = min(blockIdx.x * chunk, n_items), hi = min(lo + chunk, n_items);
  for (int t0 = lo; t0 < hi; t0 += kPlaceTile) {
    const int t1 = min(t0 + kPlaceTile, hi);
    if (threadIdx.x < kGjkBins) count[threadIdx.x] = 0;
    __syncthreads();
    // uniform trip count: every lane of a warp takes part in the matches
    for (int k0 = t0; k0 < t1; k0 += blockDim.x) {
      const int k = k0 + threadIdx.x;
      int b = -1;
      if (k < t1) {
        const int4 item = a.work[k];
        if (needs_gjk(a, item)) b = gjk_bin(a, item);
        tile_bin[k - t0] = (signed char)b;
      }
      const unsigned peers = __match_any_sync(full, b);
      if (b >= 0 && (peers & lt) == 0) atomicAdd(&count[b], __popc(peers));
    }
    __syncthreads();
    if (threadIdx.x < kGjkBins) {
      const int c = count[threadIdx.x];
      cursor[threadIdx.x] = c ? base[threadIdx.x] + atomicAdd(&a.gjk_bins[kGjkBins + threadIdx.x], c) : 0;
    }
    __syncthreads();
    for (int k0 = t0; k0 < t1; k0 += blockDim.x) {
      const int k = k0 + threadIdx.x;
      const int b = k < t1 ? tile_bin[k - t0] : -1;
      const unsigned peers = __match_any_sync(full, b);
      const int leader = __ffs(peers) - 1;
      int first = 0;
      if (b >= 0 && (peers & lt) == 0) first = atomicAdd(&cursor[b], __popc(peers));
      first = __shfl_sync(full, first, leader);
      if (b >= 0) a.gjk_order[first + __popc(peers & lt)] = k;
    }
    __syncthreads();  // count, cursor and tile_bin are reused by the next tile
  }
}

// Starting a run (the bodies, the history, the first iterate) costs about as
// much as two GJK iterations and diverges across the shapes, so lanes whose
// run has ended wait until GG_GJK_BATCH lanes of the warp are idle (by default
// the whole warp) and start their next runs together (settled drum, pair phase
// per step: 3.05 ms with batches of 16, 2.88 with 24, 2.75 with 32).
// The arrays of each thread's run (sub-determinants, dot products, simplex and
// support points: 672 bytes) live in shared memory, interleaved across the
// block's 64 threads; in local memory they overflowed L1 and were written back
// to DRAM (1.9 GB per launch on the settled drum).
constexpr int kGjkBlock = 64;
// idle lanes of a warp that wait before they write their results and start
// their next runs together
#ifndef GG_GJK_BATCH
#define GG_GJK_BATCH 32
#endif
#ifndef GG_GJK_MIN_BLOCKS
#define GG_GJK_MIN_BLOCKS 1
#endif
template <typename R>
__global__ void __launch_bounds__(kGjkBlock, GG_GJK_MIN_BLOCKS) gjk_kernel(StepArgs<R> a) {
  __shared__ double words[kGjkWords * kGjkBlock];
  const unsigned full = 0xffffffffu;
  int n_items = 0;  // GJK items: the total of the shape-pair bins
  for (int b = 0; b < kGjkBins; ++b) n_items += a.gjk_bins[b];
  unsigned long long ngjk = 0, nit = 0;
  GjkLane<R> L;
  L.run.g.base = words + threadIdx.x;
  L.run.g.stride = kGjkBlock;
  bool busy = gjk_lane_start(a, n_items, L);
  bool ended = false;    // the lane's run has ended and waits for its results to be written
  bool drained = !busy;  // no work item is left for this lane
  for (;;) {
    if (busy && gjk_iterate(L.run, L.la, L.lb)) {
      busy = false;
      ended = true;
    }
    const unsigned waiting = __ballot_sync(full, !busy && !drained);
    const unsigned running = __ballot_sync(full, busy);
    if (!waiting && !running) break;
    if (__popc(waiting) >= GG_GJK_BATCH || !running) {
      // the ended runs' results and the next runs' starts, together
      if (ended) {
        gjk_lane_finish(a, L, ngjk, nit);
        ended = false;
      }
      if (!busy && !drained) {
        busy = gjk_lane_start(a, n_items, L);
        drained = !busy;
      }
    }
  }
  warp_add(&a.stats->n_gjk_calls, ngjk);
  warp_add(&a.stats->n_gjk_iters, nit);
}

// work items [first, n_items) with the given stride; `padded`: a bound with a
// uniform trip count for the warp reductions of the statistics
template <typename R, bool DIAG, bool CONVEX, bool SV = false, bool GEOM = false>
__device__ __forceinline__ void pairs_range(const StepArgs<R>& a, int first, int stride, R dt) {
  const int n_items = (int)min((long long)*(volatile int*)a.work_n, (long long)a.n * a.clist_cap);
  const int padded = (n_items + stride - 1) / stride * stride;
  ForceStats fs{0, 0, 0, 0, 0., 0.};
  for (int k = first; k < padded; k += stride)
    if (k < n_items) pair_one<R, DIAG, CONVEX, SV, GEOM>(a, k, a.work[k], dt, fs);
  flush_force_stats(a.stats, fs);
}

// blocks per SM the register allocation of the sphere kernels must allow:
// four (128 registers, 16 warps per SM) instead of the three that 162
// registers leave; the few spills cost less than the latency the extra warps
// hide (settled 200k bed: pair phase 0.147 -> 0.137 ms mixed, 0.200 -> 0.169
// ms FP64)
#ifndef GG_PAIRS_MIN_BLOCKS
#define GG_PAIRS_MIN_BLOCKS 4
#endif
// the convex pair kernel that reads the GJK kernel's contact features at three
// blocks per SM: 170 registers without spills (settled drum, pair phase 2.56
// -> 2.50 ms per step)
#ifndef GG_PAIRS_CONVEX_MIN_BLOCKS
#define GG_PAIRS_CONVEX_MIN_BLOCKS 3
#endif
template <typename R, bool DIAG, bool CONVEX, bool SV = false, bool GEOM = false>
__global__ void __launch_bounds__(128, CONVEX ? (GEOM ? GG_PAIRS_CONVEX_MIN_BLOCKS : 1) : GG_PAIRS_MIN_BLOCKS)
    pairs_kernel(StepArgs<R> a, R dt) {
  pairs_range<R, DIAG, CONVEX, SV, GEOM>(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, dt);
}

// C. the torsor of particle s: InitializeForces(withWeight) (torsor = weight,
// Particle.cpp:1409-1416) then every contact in list order; the coordination
// number; the owner's next memory row packed: an owned entry whose result flag
// is 3 stored its memory at its rank, the others left a hole, and the kept
// entries move down over the holes (rows without holes are not touched).  The
// results of four entries are loaded at a time.
template <typename R>
__device__ __forceinline__ void sum_one(const StepArgs<R>& a, int s, V3<R>* f_out = nullptr,
                                        V3<R>* t_out = nullptr) {
  const ParticleArrays<R>& P = a.cur;
  const int sysi = P.meta[s].w;
  const double4 md = P.md[s];
  // Particle::computeWeight (Particle.cpp:414-419): mass * (1 - rho_f / rho_p) * g
  const double mass = md.x * (1. - md.w);
  const int row = P.orig[s];
  const SysDev& S = a.sys[sysi];
  V3<R> F = v3<R>(R(S.gx * mass), R(S.gy * mass), R(S.gz * mass));
  V3<R> T = v3<R>(R(0), R(0), R(0));
  const int cnt = a.ccount[s];
  const size_t base = (size_t)s * a.clist_cap;
  const int* list = a.clist + base;
  HistEntry<R>* h = a.hist_next + (size_t)row * a.hist_cap;
  int ncontact = 0, owned = 0, kept = 0;
  for (int q0 = 0; q0 < cnt; q0 += 4) {
    R4<R> rf[4], rt[4];
    int e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool in = q0 + u < cnt;
      if (in) {
        rf[u] = a.res_f[base + q0 + u];
        rt[u] = a.res_t[base + q0 + u];
        e[u] = list[q0 + u];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (q0 + u >= cnt) break;
      if (entry_owned(e[u])) {
        const int rank = owned++;
        if (rank < a.hist_cap && rf[u].w == R(3)) {
          if (kept != rank) h[kept] = h[rank];
          ++kept;
        }
      }
      if (rf[u].w == R(0)) continue;
      F = F + ld3<R>(rf[u]);
      T = T + ld3<R>(rt[u]);
      ++ncontact;
    }
  }
  if (a.hydro) {
    // AppPRSHydroFT::ComputeForces (Fluid/src/AppPRSHydroFT.cpp:29-45): the
    // fluid's force and torque, after the contacts (the collision App comes
    // first in Grains::m_allApp)
    const double* h = a.hydro + 6 * (size_t)row;
    F = F + v3<R>(R(h[0]), R(h[1]), R(h[2]));
    T = T + v3<R>(R(h[3]), R(h[4]), R(h[5]));
  }
  a.coord[s] = ncontact;
  a.hist_n_next[row] = kept;
  if (a.gjk_history) a.gdir_n_next[row] = owned < a.hist_cap ? owned : a.hist_cap;
  P.F[s] = st3<R>(F);
  P.T[s] = st3<R>(T);
  if (f_out) *f_out = F;
  if (t_out) *t_out = T;
}

// KICK: the particle's torsor is final here, and the rest of the step needs no
// other particle: the second half kick of this step and the first half kick,
// drift and binning of the next (kick_move_kernel's work) follow in the same
// thread, without the torsor's round trip through memory and a launch.
template <typename R, bool KICK = false>
__global__ void __launch_bounds__(256) sums_kernel(StepArgs<R> a, R dt_half, double dt) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) {
    *a.work_n = 0;
    if (a.gjk_next) *a.gjk_next = 0;
  }
  if (s >= a.n) return;
  V3<R> F, T;
  sum_one(a, s, &F, &T);
  if (KICK) integrate(a, a.cur, a.cur, s, F, T, 1, dt_half, 1, dt_half, dt);
}

template <typename R>
__global__ void zero_kdelta_kernel(StepArgs<R> a) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  int row = a.cur.orig[s];
  int n = a.hist_n_prev[row];
  for (int k = 0; k < n; ++k) {
    HistEntry<R>& e = a.hist_prev[(size_t)row * a.hist_cap + k];
    e.kd[0] = e.kd[1] = e.kd[2] = R(0);
    e.sp[0] = e.sp[1] = e.sp[2] = R(0);
  }
}

// overwrite the kinematic state from upload-order arrays on the device
// (ParticleKinematics::setAngularVelocity gives the body-frame rate)
template <typename R>
__device__ __forceinline__ void set_kinematics(const StepArgs<R>& a, int s, const KinematicStage& st, size_t i) {
  const ParticleArrays<R>& P = a.cur;
  double4 xr = P.xr[s];
  xr.x = st.position[3 * i];
  xr.y = st.position[3 * i + 1];
  xr.z = st.position[3 * i + 2];
  P.xr[s] = xr;
  const double* qi = st.quaternion + 4 * i;
  P.q[s] = make_double4(qi[0], qi[1], qi[2], qi[3]);
  P.v[s] = st3<R>(v3<R>(R(st.velocity[3 * i]), R(st.velocity[3 * i + 1]), R(st.velocity[3 * i + 2])));
  Qt<double> q{v3<double>(qi[0], qi[1], qi[2]), qi[3]};
  V3<double> w = v3<double>(st.omega[3 * i], st.omega[3 * i + 1], st.omega[3 * i + 2]);
  P.w[s] = st3<R>(v3<R>(R(w.x), R(w.y), R(w.z)));
  V3<double> wbf = q_to_body(q, w);
  P.wbf[s] = st3<R>(v3<R>(R(wbf.x), R(wbf.y), R(wbf.z)));
  if (a.has_basis && st.basis)
    for (int k = 0; k < 9; ++k) P.basis[9 * (size_t)s + k] = st.basis[9 * i + k];
}

template <typename R>
__global__ void update_dynamic_kernel(StepArgs<R> a, KinematicStage st) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  set_kinematics(a, s, st, (size_t)a.cur.orig[s]);
}

// translational and angular velocities (world frame, upload order) of every
// particle; the body-frame angular velocity follows from the quaternion
// (ParticleKinematics::setAngularVelocity, ParticleKinematics.cpp:197-203)
template <typename R>
__global__ void set_velocities_kernel(StepArgs<R> a, const double* vel, const double* omega) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const ParticleArrays<R>& P = a.cur;
  const size_t i = (size_t)P.orig[s];
  P.v[s] = st3<R>(v3<R>(R(vel[3 * i]), R(vel[3 * i + 1]), R(vel[3 * i + 2])));
  const double4 qd = P.q[s];
  Qt<double> q{v3<double>(qd.x, qd.y, qd.z), qd.w};
  V3<double> w = v3<double>(omega[3 * i], omega[3 * i + 1], omega[3 * i + 2]);
  P.w[s] = st3<R>(v3<R>(R(w.x), R(w.y), R(w.z)));
  V3<double> wbf = q_to_body(q, w);
  P.wbf[s] = st3<R>(v3<R>(R(wbf.x), R(wbf.y), R(wbf.z)));
}

// rho_f / rho_p of every particle (upload order) into md.w of the current arrays
template <typename R>
__global__ void set_fluid_ratio_kernel(StepArgs<R> a, const double* ratio) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < a.n) a.cur.md[s].w = ratio[a.cur.orig[s]];
}

// slot of every upload index (the inverse of orig)
template <typename R>
__global__ void slot_of_row_kernel(StepArgs<R> a, int* slot_of) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < a.n) slot_of[a.cur.orig[s]] = s;
}

// the kinematic state of the listed upload indices (stage entry k for rows[k])
template <typename R>
__global__ void update_rows_kernel(StepArgs<R> a, KinematicStage st, const long long* rows, long long n_rows,
                                   const int* slot_of) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n_rows) set_kinematics(a, slot_of[rows[k]], st, (size_t)k);
}

// the state in upload order, one array per field (any may be null): the
// device side of grains_gpu_download_particles.  Spheres without a stored
// basis get the rotation matrix of their quaternion.
template <typename R>
__global__ void pack_download_kernel(StepArgs<R> a, DownloadStage d) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const ParticleArrays<R>& P = a.cur;
  const size_t i = (size_t)P.orig[s];
  const double4 xr = P.xr[s], q = P.q[s];
  if (d.position) {
    d.position[3 * i] = xr.x;
    d.position[3 * i + 1] = xr.y;
    d.position[3 * i + 2] = xr.z;
  }
  if (d.quaternion) {
    d.quaternion[4 * i] = q.x;
    d.quaternion[4 * i + 1] = q.y;
    d.quaternion[4 * i + 2] = q.z;
    d.quaternion[4 * i + 3] = q.w;
  }
  if (d.basis) {
    if (a.has_basis) {
      for (int k = 0; k < 9; ++k) d.basis[9 * i + k] = P.basis[9 * (size_t)s + k];
    } else {
      const double x = q.x, y = q.y, z = q.z, w0 = q.w;
      const double m[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w0 * z), 2 * (x * z + w0 * y),
                           2 * (x * y + w0 * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w0 * x),
                           2 * (x * z - w0 * y), 2 * (y * z + w0 * x), 1 - 2 * (x * x + y * y)};
      for (int k = 0; k < 9; ++k) d.basis[9 * i + k] = m[k];
    }
  }
  const R4<R> v = P.v[s], w = P.w[s], F = P.F[s], T = P.T[s];
  if (d.velocity) {
    d.velocity[3 * i] = double(v.x);
    d.velocity[3 * i + 1] = double(v.y);
    d.velocity[3 * i + 2] = double(v.z);
  }
  if (d.omega) {
    d.omega[3 * i] = double(w.x);
    d.omega[3 * i + 1] = double(w.y);
    d.omega[3 * i + 2] = double(w.z);
  }
  if (d.force) {
    d.force[3 * i] = double(F.x);
    d.force[3 * i + 1] = double(F.y);
    d.force[3 * i + 2] = double(F.z);
  }
  if (d.torque) {
    d.torque[3 * i] = double(T.x);
    d.torque[3 * i + 1] = double(T.y);
    d.torque[3 * i + 2] = double(T.z);
  }
  if (d.coordination) d.coordination[i] = a.coord[s];
  if (d.id) d.id[i] = P.meta[s].x;
}

// Imposed motion of one obstacle over the step ending at T
// (ObstacleKinematicsVelocity::ImposedMotion, ObstacleKinematicsVelocity.cpp:
// 86-122, with ObstacleImposedVelocity::isActif / isCompleted /
// translationalMotion / angularMotion / translationalVelocity / angularVelocity,
// ObstacleImposedVelocity.cpp:306-455), then SimpleObstacle::Move
// (SimpleObstacle.cpp:119-170): the active loadings' motions add up; an
// obstacle that did not move keeps its velocities and its box.  Then the
// world AABB (Convex::bbox, Convex.cpp:29-41 -> BBox::setValue, BBox.cpp:235-239).
static __device__ V3<double> loading_motion(const LoadingDev& L, double T, double dt, double sub, V3<double> cg) {
  const double td = xsub(T, dt);
  const double ti = td < L.ts ? L.ts : td;
  const double te = T > L.te ? L.te : T;
  const V3<double> u = v3<double>(L.unit[0], L.unit[1], L.unit[2]);
  switch (L.type) {
    case GRAINS_GPU_CONSTANT_TRANSLATION:
      return v3<double>(L.vel[0] * sub, L.vel[1] * sub, L.vel[2] * sub);
    case GRAINS_GPU_CRENEL_TRANSLATION:
      return sc(u, L.amp * (int((0.5 * (ti + te) - L.ts) / L.period) % 2 == 0 ? 1 : -1) * sub);
    case GRAINS_GPU_SIN_TRANSLATION:
      return sc(u, (L.amp * L.period / (2. * kPi)) * (cos(2. * kPi * (ti - L.ts) / L.period + L.phase) -
                                                       cos(2. * kPi * (te - L.ts) / L.period + L.phase)));
    case GRAINS_GPU_MULTISIN_TRANSLATION: {
      double m[3];
      for (int i = 0; i < 3; ++i)
        m[i] = (L.mamp[i] * L.mper[i] / (2. * kPi)) * (cos(2. * kPi * (ti - L.ts) / L.mper[i] + L.mphase[i]) -
                                                        cos(2. * kPi * (te - L.ts) / L.mper[i] + L.mphase[i])) *
               L.unit[i];
      return v3<double>(m[0], m[1], m[2]);
    }
    case GRAINS_GPU_CONSTANT_ROTATION: {
      if (!L.has_center) return v3<double>(0., 0., 0.);
      const V3<double> rota = sc(v3<double>(L.omega[0], L.omega[1], L.omega[2]), sub);
      const double d = norm(rota);
      Qt<double> q{v3<double>(0., 0., 0.), 1.};
      if (d != 0.) q = Qt<double>{sc(rota, sin(d / 2.) / d), cos(d / 2.)};
      const V3<double> rel = cg - v3<double>(L.center[0], L.center[1], L.center[2]);
      return q_rotate(q, rel) - rel;
    }
  }
  return v3<double>(0., 0., 0.);
}

static __device__ V3<double> loading_velocity(const LoadingDev& L, double T, double dt, V3<double> cg) {
  if (T > L.te + dt * 1.e-5) return v3<double>(0., 0., 0.);  // isCompleted
  const V3<double> u = v3<double>(L.unit[0], L.unit[1], L.unit[2]);
  switch (L.type) {
    case GRAINS_GPU_CONSTANT_TRANSLATION:
      return v3<double>(L.vel[0], L.vel[1], L.vel[2]);
    case GRAINS_GPU_SIN_TRANSLATION:
      return sc(u, L.amp * sin(2. * kPi * (T - L.ts) / L.period + L.phase));
    case GRAINS_GPU_CRENEL_TRANSLATION:
      return sc(u, L.amp * (int((T - L.ts) / L.period) % 2 == 0 ? 1 : -1));
    case GRAINS_GPU_MULTISIN_TRANSLATION: {
      double v[3];
      for (int i = 0; i < 3; ++i) v[i] = L.mamp[i] * sin(2. * kPi * (T - L.ts) / L.mper[i] + L.mphase[i]) * L.unit[i];
      return v3<double>(v[0], v[1], v[2]);
    }
    case GRAINS_GPU_CONSTANT_ROTATION:
      return L.has_center ? cross(v3<double>(L.omega[0], L.omega[1], L.omega[2]),
                                  cg - v3<double>(L.center[0], L.center[1], L.center[2]))
                          : v3<double>(0., 0., 0.);
  }
  return v3<double>(0., 0., 0.);
}

// ObstacleImposedVelocity::isActif (ObstacleImposedVelocity.cpp:306-315) over [T - dt, T]
static __device__ __forceinline__ bool loading_active(const LoadingDev& L, double T, double dt, double& sub) {
  const double td = xsub(T, dt);
  sub = xsub(T, td);
  if (td < L.ts) sub = xsub(sub, xsub(L.ts, td));
  if (L.te < T) sub = xsub(sub, xsub(T, L.te));
  return sub > dt * 1.e-5;
}

static __device__ void obstacle_aabb(ObstacleDev& O, const ShapeDev* shapes, const double* verts);

// returns whether the obstacle moved
static __device__ __noinline__ bool obstacle_move_one(ObstacleDev& O, const LoadingDev* loads, const ShapeDev* shapes,
                                                      const double* verts, double T, double dt) {
  const V3<double> cg = v3<double>(O.o[0], O.o[1], O.o[2]);
  V3<double> depl = v3<double>(0., 0., 0.), rota = depl, vt = depl, vr = depl;
  for (int k = O.load_first; k < O.load_first + O.load_count; ++k) {
    const LoadingDev& L = loads[k];
    double sub;
    if (!loading_active(L, T, dt, sub)) continue;
    depl = depl + loading_motion(L, T, dt, sub, cg);
    const V3<double> om = v3<double>(L.omega[0], L.omega[1], L.omega[2]);
    if (L.type == GRAINS_GPU_CONSTANT_ROTATION) rota = rota + sc(om, sub);
    vt = vt + loading_velocity(L, T, dt, cg);
    if (L.type == GRAINS_GPU_CONSTANT_ROTATION && !(T > L.te + dt * 1.e-5)) vr = vr + om;
  }
  const double d = norm(rota);
  if (!(norm(depl) != 0. || d != 0.)) return false;
  Qt<double> qrot{v3<double>(0., 0., 0.), 1.};
  if (d != 0.) qrot = Qt<double>{sc(rota, sin(d / 2.) / d), cos(d / 2.)};
  const Qt<double> qdt = qmul(qrot, Qt<double>{v3<double>(0., 0., 0.), 1.});
  M3 b;
  for (int t = 0; t < 9; ++t) b.m[t] = O.b[t];
  O.o[0] = cg.x + depl.x;
  O.o[1] = cg.y + depl.y;
  O.o[2] = cg.z + depl.z;
  mrotate_left(b, qdt);
  for (int t = 0; t < 9; ++t) O.b[t] = b.m[t];
  O.vel[0] = vt.x;
  O.vel[1] = vt.y;
  O.vel[2] = vt.z;
  O.omega[0] = vr.x;
  O.omega[1] = vr.y;
  O.omega[2] = vr.z;
  obstacle_aabb(O, shapes, verts);
  return true;
}

// the obstacle's world bounding box from its pose (Component::BoundingBox)
static __device__ void obstacle_aabb(ObstacleDev& O, const ShapeDev* shapes, const double* verts) {
  M3 b;
  for (int t = 0; t < 9; ++t) b.m[t] = O.b[t];
  const ShapeDev& sh = shapes[O.shape];
  LocalBody<double> L{};
  L.type = sh.type;
  L.nverts = sh.nverts;
  L.verts = verts + 3 * sh.vert_offset;
  L.radius = sh.radius;
  L.cyl_r = sh.radius;
  L.cyl_hh = sh.half_height;
  L.ext = v3<double>(sh.ext[0], sh.ext[1], sh.ext[2]);
  double mn[3], mx[3];
  for (int i = 0; i < 3; ++i) {
    const D3 r = mrow(b, i);
    const V3<double> rv = v3<double>(r.x, r.y, r.z);
    const V3<double> sp = support_local(L, rv), sn = support_local(L, -rv);
    mn[i] = xadd(O.o[i], xdot(r, d3(sn.x, sn.y, sn.z)));
    mx[i] = xadd(O.o[i], xdot(r, d3(sp.x, sp.y, sp.z)));
  }
  for (int i = 0; i < 3; ++i) {
    O.bbe[i] = xdiv(xsub(mx[i], mn[i]), 2.);
    O.bbc[i] = xadd(mn[i], O.bbe[i]);
  }
}


// ObstacleImposedForce::translationalVelocity (ObstacleImposedForce.cpp:183-252),
// "ConstantTranslation": a PID controller (Ziegler-Nichols coefficients from
// the virtual mass) on the difference between the contact force F on the
// obstacle and the imposed force, along the force's direction.  pid: the
// system's history (the reference's static variables, shared by all its
// imposed forces).  vt, trans: the force kinematics' velocity and its
// translation over the active part `sub` of the step.
static __device__ void force_velocity(const ObstacleDev& O, const LoadingDev& L, const double F[3], double* pid,
                                      double T, double dt, double sub, double vt[3], double trans[3]) {
  const V3<double> famp = v3<double>(L.vel[0], L.vel[1], L.vel[2]);
  const double mass = L.amp > 0. ? L.amp : dt * dt * norm(famp) * 1.e7 / (2. * O.crust);
  const double Kp = 0.5 * dt * dt / mass;
  const double Ki = 2. * Kp / dt;
  const double Kd = 3. * Kp * dt / 24.;
  if (pid[9] == 0.) pid[9] = norm(v3<double>(F[0], F[1], F[2])) > kEpsilon ? 1. : 0.;
  const double fa[3] = {famp.x, famp.y, famp.z};
  double df[3];
  for (int i = 0; i < 3; ++i) df[i] = (F[i] - fa[i]) * L.unit[i];
  if (pid[9] != 0.) {
    const double c0 = Kp + Ki * dt + Kd / dt, c1 = Kp + 2. * Kd / dt, c2 = Kd / dt;
    for (int i = 0; i < 3; ++i) {
      const double depl = pid[6 + i] + df[i] * c0 - pid[i] * c1 + pid[3 + i] * c2;
      vt[i] = depl / dt;
      trans[i] = depl * (sub / dt);
      pid[3 + i] = pid[i];
      pid[i] = df[i];
      pid[6 + i] = depl;
    }
  } else {
    for (int i = 0; i < 3; ++i) {
      vt[i] = L.unit[i] * (-L.period);
      trans[i] = vt[i] * sub;
    }
  }
  if (T > L.te + dt * 1.e-5)  // isCompleted
    for (int i = 0; i < 3; ++i) vt[i] = 0.;
}

// Imposed motion of every moving obstacle over one step, by one block: every
// thread reads the clock before thread 0 advances it.
// AllComponents::Move (AllComponents.cpp:168-213): when a loading of a system
// is active over [T - dt, T], or was over the previous step, the velocities of
// the system's obstacles are reset (Obstacle::resetKinematics, Obstacle.cpp:
// 160-167); when one is active, its obstacles move.  Global flags per system:
// [2 s] active now, [2 s + 1] active over the previous step.
static __device__ __forceinline__ void obstacle_move_block(ObstacleDev* obs, const int* moving_idx, int n_moving,
                                                           const LoadingDev* loads, int* flags, int n_sys,
                                                           const ShapeDev* shapes, const double* verts, double dt,
                                                           double* clock, double host_time, int use_host_time,
                                                           const double* force_part = nullptr,
                                                           double* force_pid = nullptr) {
  const double T = use_host_time ? host_time : xadd(*clock, dt);
  __syncthreads();
  if (threadIdx.x == 0) *clock = T;
  for (int s = threadIdx.x; s < n_sys; s += blockDim.x) flags[2 * s] = 0;
  __syncthreads();
  for (int u = threadIdx.x; u < n_moving; u += blockDim.x) {
    const ObstacleDev& O = obs[moving_idx[u]];
    bool any = false;
    for (int k = O.load_first; k < O.load_first + O.load_count && !any; ++k) {
      double sub;
      any = loading_active(loads[k], T, dt, sub);
    }
    if (any) flags[2 * O.sys] = 1;
  }
  __syncthreads();
  for (int u = threadIdx.x; u < n_moving; u += blockDim.x) {
    ObstacleDev& O = obs[moving_idx[u]];
    const int now = flags[2 * O.sys], before = flags[2 * O.sys + 1];
    if (now || before)
      for (int i = 0; i < 3; ++i) {
        O.vel[i] = 0.;
        O.omega[i] = 0.;
      }
    O.moved = now ? (obstacle_move_one(O, loads, shapes, verts, T, dt) ? 1 : 0) : 0;
  }
  __syncthreads();
  // the imposed forces (ObstacleKinematicsForce::ImposedMotion, ObstacleKinematicsForce.cpp:
  // 64-92, and SimpleObstacle::Move, SimpleObstacle.cpp:146-166): in obstacle order, one
  // thread, since the controller history is shared; every active force loading updates the
  // kinematics in turn, the obstacle moves when the resulting velocity is not zero, and its
  // velocity adds the force kinematics' velocity (Obstacle::setVelocity, Obstacle.cpp:635-640)
  if (force_part && threadIdx.x == 0)
    for (int u = 0; u < n_moving; ++u) {
      ObstacleDev& O = obs[moving_idx[u]];
      if (O.force_slot < 0 || !flags[2 * O.sys]) continue;
      double F[3] = {0., 0., 0.};
      for (int b = 0; b < kForceBlocks; ++b)
        for (int i = 0; i < 3; ++i) F[i] += force_part[(b * kMaxForceObstacles + O.force_slot) * 3 + i];
      double vt[3] = {0., 0., 0.}, tr[3] = {0., 0., 0.};
      for (int k = O.load_first; k < O.load_first + O.load_count; ++k) {
        double sub;
        if (loads[k].type != GRAINS_GPU_FORCE_TRANSLATION || !loading_active(loads[k], T, dt, sub)) continue;
        force_velocity(O, loads[k], F, force_pid + kForcePidWords * O.sys, T, dt, sub, vt, tr);
      }
      const bool move = norm(v3<double>(vt[0], vt[1], vt[2])) != 0.;
      if (move) {
        for (int i = 0; i < 3; ++i) O.o[i] = O.o[i] + tr[i];
        obstacle_aabb(O, shapes, verts);
      }
      if (move || O.moved)
        for (int i = 0; i < 3; ++i) O.vel[i] = O.vel[i] + vt[i];
    }
  __syncthreads();
  for (int s = threadIdx.x; s < n_sys; s += blockDim.x) flags[2 * s + 1] = flags[2 * s];
}

#ifdef GG_DEFINE_SHARED_KERNELS
// Imposed obstacle motion of one step (ObstacleKinematicsVelocity::ImposedMotion,
// ObstacleKinematicsVelocity.cpp:86-122; ObstacleImposedVelocity.cpp:388-445).
// The clock is the reference's m_time: T = clock + dt, and the motion acts over
// the sub-interval T - (T - dt) (ObstacleImposedVelocity::isActif, :306-315).
// With use_host_time the caller gives T directly.  One block: every thread
// reads the clock before thread 0 advances it.
__global__ void obstacle_move_kernel(ObstacleDev* obs, const int* moving_idx, int n_moving, const LoadingDev* loads,
                                     int* flags, int n_sys, const ShapeDev* shapes, const double* verts, double dt,
                                     double* clock, double host_time, int use_host_time, const double* force_part,
                                     double* force_pid) {
  obstacle_move_block(obs, moving_idx, n_moving, loads, flags, n_sys, shapes, verts, dt, clock, host_time,
                      use_host_time, force_part, force_pid);
}

#endif  // GG_DEFINE_SHARED_KERNELS

// candidate pairs (diagnostic): pairs with both cells equal or adjacent
template <typename R>
__global__ void candidate_pairs_kernel(StepArgs<R> a, int sys, int include_obstacles, int* out, int cap,
                                       unsigned long long* count) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const ParticleArrays<R>& P = a.cur;
  const int4 mi = P.meta[s];
  if (mi.w != sys) return;
  const double4 xi = P.xr[s];
  const SysDev& S = a.sys[mi.w];
  int ci, cj, ck;
  cell_of(S, xi.x, xi.y, xi.z, ci, cj, ck);
  const int i0 = max(ci - 1, 0), i1 = min(ci + 1, S.nbi - 1);
  for (int dj = -1; dj <= 1; ++dj) {
    const int j = cj + dj;
    if (j < 0 || j >= S.nbj) continue;
    for (int dk = -1; dk <= 1; ++dk) {
      const int k = ck + dk;
      if (k < 0 || k >= S.nbk) continue;
      const int t0 = a.cell_start[cell_index(S, i0, j, k)];
      const int t1 = a.cell_start[cell_index(S, i1, j, k) + 1];
      for (int t = t0; t < t1; ++t) {
        const int j = a.perm[t];
        int idj = P.meta[j].x;
        if (j == s || !(mi.x < idj)) continue;
        unsigned long long slot = atomicAdd(count, 1ull);
        if (slot < (unsigned long long)cap) {
          out[2 * slot] = mi.x;
          out[2 * slot + 1] = idj;
        }
      }
    }
  }
  if (include_obstacles) {
    const int cell = cell_index(S, ci, cj, ck);
    const D3 cg = d3(xadd(xadd(S.ox, xmul(double(ci), S.ex)), xdiv(S.ex, 2.)),
                     xadd(xadd(S.oy, xmul(double(cj), S.ey)), xdiv(S.ey, 2.)),
                     xadd(xadd(S.oz, xmul(double(ck), S.ez)), xdiv(S.ez, 2.)));
    for (int u = a.cell_obs_start[cell]; u < a.cell_obs_start[cell + 1]; ++u) {
      unsigned long long slot = atomicAdd(count, 1ull);
      if (slot < (unsigned long long)cap) {
        out[2 * slot] = mi.x;
        out[2 * slot + 1] = a.obs[a.cell_obs_idx[u]].id;
      }
    }
    for (int u = 0; u < S.n_moving; ++u) {
      const ObstacleDev& O = a.obs[a.moving_idx[S.moving_offset + u]];
      if (!in_zone(d3(O.bbc[0], O.bbc[1], O.bbc[2]), d3(O.bbe[0], O.bbe[1], O.bbe[2]), cg, S.ex, S.ey, S.ez))
        continue;
      unsigned long long slot = atomicAdd(count, 1ull);
      if (slot < (unsigned long long)cap) {
        out[2 * slot] = mi.x;
        out[2 * slot + 1] = O.id;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// launchers
inline int grid_for(long long n, int block) { return (int)((n + block - 1) / block); }

inline int check_launch() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : GRAINS_GPU_CUDA_ERROR;
}

template <typename R>
int launch_kick_move(const StepArgs<R>& a, cudaStream_t s, int do_kick2, double dt_kick2, int do_move, double dt_v,
                     double dt_x) {
  if (a.n == 0) return 0;
  kick_move_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a, do_kick2, R(dt_kick2), do_move, R(dt_v), dt_x);
  return check_launch();
}

template <typename R>
int launch_bin(const StepArgs<R>& a, cudaStream_t s) {
  if (a.n == 0) return 0;
  bin_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a);
  return check_launch();
}

template <typename R>
int launch_sort_and_gather(const StepArgs<R>& a, cudaStream_t s, int gather, int gather_forces) {
  const int C = a.n_cells;
  const int nb = grid_for(C, kScanTile);
  if (nb > kMaxScanTiles) return GRAINS_GPU_INVALID_ARGUMENT;
  scan_tiles_kernel<<<nb, kScanThreads, 0, s>>>(a.cell_count, a.cell_cursor, a.block_sums, C);
  if (a.n > 0) scatter_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a);
  cell_sort_kernel<R><<<grid_for(C, kCellSortThreads), kCellSortThreads, 0, s>>>(a);
  if (a.n > 0 && gather) gather_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a, gather_forces);
  return check_launch();
}

// the GJK kernel keeps every SM full: its resident blocks per SM x the SMs
template <typename R>
int gjk_grid() {
  static int grid = 0;
  if (!grid) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // as much shared memory as the SM has, for the runs' arrays
    cudaFuncSetAttribute(gjk_kernel<R>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gjk_kernel<R>, kGjkBlock, 0);
    grid = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }
  return grid;
}

template <typename R>
int launch_forces(const StepArgs<R>& a, cudaStream_t s, double dt, int diag, int phases, int kick) {
  if (a.n == 0) return 0;
  const int cb = (a.contacts_block >= 32 && a.contacts_block <= 256) ? a.contacts_block : 256;
  const int fb = (a.forces_block >= 32 && a.forces_block <= 128) ? a.forces_block : 128;
  if (phases & 1) contacts_kernel<R><<<grid_for(a.n, cb), cb, 0, s>>>(a);
  if (!(phases & 6)) return check_launch();
  auto sums = [&]() {
    if (kick)
      sums_kernel<R, true><<<grid_for(a.n, 256), 256, 0, s>>>(a, R(0.5 * dt), dt);
    else
      sums_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a, R(0), 0.);
  };
  if (!(phases & 2)) {
    sums();
    return check_launch();
  }
  // about two work items per thread in a settled packing; the grid-stride
  // loop takes any count
  const int g = (int)std::min<long long>(grid_for(2ll * a.n, fb), 1ll << 20);
  if (a.has_convex && a.gjk_sv) {  // the signed-volume GJK: a kernel of its own
    if (diag)
      pairs_kernel<R, true, true, true><<<g, fb, 0, s>>>(a, R(dt));
    else
      pairs_kernel<R, false, true, true><<<g, fb, 0, s>>>(a, R(dt));
  } else if (a.has_convex && a.gjk_out) {  // the GJK items grouped by shape pair, the GJK kernel, the law
    cudaMemsetAsync(a.gjk_bins, 0, 2 * kGjkBins * sizeof(int), s);
    const int gb = 2 * 148;
    gjk_count_kernel<R><<<gb, 256, 0, s>>>(a);
    gjk_place_kernel<R><<<gb, 256, 0, s>>>(a);
    gjk_kernel<R><<<gjk_grid<R>(), kGjkBlock, 0, s>>>(a);
    if (diag)
      pairs_kernel<R, true, true, false, true><<<g, fb, 0, s>>>(a, R(dt));
    else
      pairs_kernel<R, false, true, false, true><<<g, fb, 0, s>>>(a, R(dt));
  } else if (a.has_convex) {
    if (diag)
      pairs_kernel<R, true, true><<<g, fb, 0, s>>>(a, R(dt));
    else
      pairs_kernel<R, false, true><<<g, fb, 0, s>>>(a, R(dt));
  } else {
    if (diag)
      pairs_kernel<R, true, false><<<g, fb, 0, s>>>(a, R(dt));
    else
      pairs_kernel<R, false, false><<<g, fb, 0, s>>>(a, R(dt));
  }
  if (phases & 4) sums();
  return check_launch();
}

template <typename R>
int launch_zero_kdelta(const StepArgs<R>& a, cudaStream_t s) {
  if (a.n == 0) return 0;
  zero_kdelta_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a);
  return check_launch();
}

#ifdef GG_DEFINE_SHARED_KERNELS
int launch_obstacle_move(ObstacleDev* obs, const int* moving_idx, int n_moving, const LoadingDev* loads,
                         int* load_flags, int n_sys, const ShapeDev* shapes, const double* verts, double dt,
                         double* clock, double host_time, int use_host_time, const double* force_part,
                         double* force_pid, cudaStream_t s) {
  if (n_moving <= 0) return 0;
  obstacle_move_kernel<<<1, 256, 0, s>>>(obs, moving_idx, n_moving, loads, load_flags, n_sys, shapes, verts, dt, clock,
                                         host_time, use_host_time, force_part, force_pid);
  return check_launch();
}
#endif

// The contact forces on the force-driven obstacles (Obstacle::getForce: the
// sum of the reactions -f of the particles' contacts with the obstacle,
// HookeMemoryContactForceModel.cpp:236-238 and the other laws alike), from the
// list entries' results of the last force evaluation, summed in double:
// each thread over a fixed set of rows in list order, each block in a fixed
// tree, one partial sum per block and obstacle.
template <typename R>
__global__ void __launch_bounds__(256) obstacle_force_kernel(StepArgs<R> a, double* part, int n_obs) {
  __shared__ double red[256];
  double acc[kMaxForceObstacles * 3];
  for (int k = 0; k < kMaxForceObstacles * 3; ++k) acc[k] = 0.;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < a.n; s += gridDim.x * blockDim.x) {
    const int cnt = min(a.ccount[s], a.clist_cap);
    const size_t base = (size_t)s * a.clist_cap;
    for (int q = 0; q < cnt; ++q) {
      const int e = a.clist[base + q];
      if (e >= 0 || -1 - e >= n_obs) continue;
      const int slot = a.obs[-1 - e].force_slot;
      if (slot < 0 || slot >= kMaxForceObstacles) continue;
      const R4<R> rf = a.res_f[base + q];
      if (rf.w == R(0)) continue;
      acc[3 * slot] -= (double)rf.x;
      acc[3 * slot + 1] -= (double)rf.y;
      acc[3 * slot + 2] -= (double)rf.z;
    }
  }
  for (int k = 0; k < kMaxForceObstacles * 3; ++k) {
    red[threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x * kMaxForceObstacles * 3 + k] = red[0];
    __syncthreads();
  }
}

template <typename R>
int launch_obstacle_force(const StepArgs<R>& a, double* force_part, int n_obs, cudaStream_t s) {
  obstacle_force_kernel<R><<<kForceBlocks, 256, 0, s>>>(a, force_part, n_obs);
  return check_launch();
}

template <typename R>
int launch_update_dynamic(const StepArgs<R>& a, cudaStream_t s, const KinematicStage& st) {
  if (a.n == 0) return 0;
  update_dynamic_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a, st);
  return check_launch();
}

template <typename R>
int launch_set_velocities(const StepArgs<R>& a, cudaStream_t s, const double* vel, const double* omega) {
  if (a.n == 0) return 0;
  set_velocities_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a, vel, omega);
  return check_launch();
}

template <typename R>
int launch_set_fluid_ratio(const StepArgs<R>& a, cudaStream_t s, const double* ratio) {
  if (a.n == 0) return 0;
  set_fluid_ratio_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a, ratio);
  return check_launch();
}

template <typename R>
int launch_update_rows(const StepArgs<R>& a, cudaStream_t s, const KinematicStage& st, const long long* rows,
                       long long n_rows, int* slot_of) {
  if (a.n == 0 || n_rows == 0) return 0;
  slot_of_row_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a, slot_of);
  update_rows_kernel<R><<<(int)((n_rows + 255) / 256), 256, 0, s>>>(a, st, rows, n_rows, slot_of);
  return check_launch();
}

template <typename R>
int launch_pack_download(const StepArgs<R>& a, cudaStream_t s, const DownloadStage& d) {
  if (a.n == 0) return 0;
  pack_download_kernel<R><<<grid_for(a.n, 256), 256, 0, s>>>(a, d);
  return check_launch();
}

template <typename R>
int launch_candidate_pairs(const StepArgs<R>& a, cudaStream_t s, int sys, int include_obstacles, int* out, int cap,
                           unsigned long long* count) {
  if (a.n == 0) return 0;
  candidate_pairs_kernel<R><<<grid_for(a.n, 128), 128, 0, s>>>(a, sys, include_obstacles, out, cap, count);
  return check_launch();
}

// ---------------------------------------------------------------------------
// Persistent step: n middle steps of grains_gpu_step in ONE cooperative launch
// (every block resident), the phases separated by a grid barrier.  The same
// device bodies as the per-phase kernels run in grid-stride loops, so the
// results are bit-identical to the launched pipeline.  Measured on B200 it is
// slower than the graph-replayed launches at every size tried (1,000 spheres:
// 35.4 vs 30.9 us per step; 200,000: 127 vs 78 us): each phase is a chain of
// dependent L2 round trips whose latency a barrier does not hide any better
// than a launch boundary, and for large systems every phase runs at the
// occupancy of the heaviest (the contact law).  Kept as a tuning choice.

constexpr int kPersistentThreads = 128;
// default bound of a barrier wait: 2^24 polls x 64 ns sleep, about a second
// (StepArgs::barrier_polls; a test lowers it to make the wait run out)

// Grid barrier with a bounded wait: bar[0] counts arrivals, bar[1] is the
// generation.  A wait that runs out sets GRAINS_GPU_TIMEOUT and returns false;
// the kernel then returns, and the others run out at their next barrier.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* status, long long polls) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long it = 0;
      while (*gen == g) {
        if (++it > polls || (*((volatile int*)status) & GRAINS_GPU_TIMEOUT)) {
          ok = 0;
          atomicOr(status, GRAINS_GPU_TIMEOUT);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

template <typename R, bool CONVEX>
__global__ void __launch_bounds__(kPersistentThreads) persistent_steps_kernel(
    StepArgs<R> a0, int n_steps, R dt_r, double dt, int gather_every, int since_gather, int n_moving,
    double* clock, unsigned* bar, int* sums) {
  StepArgs<R> a = a0;  // the buffer roles change from step to step
  const int nthreads = gridDim.x * blockDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n, C = a.n_cells;
  int* status = &a.stats->status;
  __shared__ int offset_s;
  // a test of the bounded wait: this block leaves before the first barrier,
  // so that the others' waits run out
  if ((int)blockIdx.x == a.barrier_skip_block) return;
  for (int step = 0; step < n_steps; ++step) {
    // exclusive scan of the cell counts: a chunk per block, then the offsets
    {
      const int chunk = (C + gridDim.x - 1) / gridDim.x;
      const int c0 = min(C, (int)blockIdx.x * chunk), c1 = min(C, c0 + chunk);
      int run = 0;
      for (int base = c0; base < c1; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < c1 ? a.cell_count[i] : 0;
        int total;
        const int pre = block_exclusive_scan(v, &total);
        if (i < c1) a.cell_start[i] = run + pre;
        run += total;
      }
      if (threadIdx.x == 0) sums[blockIdx.x] = run;
      if (!grid_barrier(bar, status, a.barrier_polls)) return;
      if (threadIdx.x == 0) {
        int o = 0;
        for (int b = 0; b < (int)blockIdx.x; ++b) o += sums[b];
        offset_s = o;
        if (blockIdx.x == gridDim.x - 1) a.cell_start[C] = o + run;
      }
      __syncthreads();
      for (int i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
        const int v = a.cell_start[i] + offset_s;
        a.cell_start[i] = v;
        a.cell_cursor[i] = v;
      }
      if (!grid_barrier(bar, status, a.barrier_polls)) return;
    }
    for (int s = tid; s < n; s += nthreads) scatter_one(a, s);
    if (!grid_barrier(bar, status, a.barrier_polls)) return;
    for (int c = tid; c < C; c += nthreads) cell_sort_one(a, c);
    if (!grid_barrier(bar, status, a.barrier_polls)) return;
    if (since_gather + 1 >= gather_every) {
      for (int t = tid; t < n; t += nthreads) gather_one(a, t, 0);
      const ParticleArrays<R> tmp = a.cur;
      a.cur = a.alt;
      a.alt = tmp;
      since_gather = 0;
      if (!grid_barrier(bar, status, a.barrier_polls)) return;
    } else {
      ++since_gather;
    }
    contacts_range(a, tid, nthreads);
    if (!grid_barrier(bar, status, a.barrier_polls)) return;
    pairs_range<R, false, CONVEX>(a, tid, nthreads, dt_r);
    if (!grid_barrier(bar, status, a.barrier_polls)) return;
    if (tid == 0) *a.work_n = 0;  // every block has read the count
    for (int s = tid; s < n; s += nthreads) sum_one(a, s);
    {
      HistEntry<R>* h = a.hist_prev;
      a.hist_prev = a.hist_next;
      a.hist_next = h;
      int* hn = a.hist_n_prev;
      a.hist_n_prev = a.hist_n_next;
      a.hist_n_next = hn;
      GjkDir* gd = a.gdir_prev;
      a.gdir_prev = a.gdir_next;
      a.gdir_next = gd;
      int* gn = a.gdir_n_prev;
      a.gdir_n_prev = a.gdir_n_next;
      a.gdir_n_next = gn;
    }
    if (!grid_barrier(bar, status, a.barrier_polls)) return;
    for (int s = tid; s < n; s += nthreads)
      integrate(a, a.cur, a.cur, s, ld3<R>(a.cur.F[s]), ld3<R>(a.cur.T[s]), 1, R(0.5) * dt_r, 1, R(0.5) * dt_r, dt);
    if (blockIdx.x == 0 && n_moving > 0)
      obstacle_move_block(const_cast<ObstacleDev*>(a.obs), a.moving_idx, n_moving, a.loads, a.load_flags, a.n_sys,
                          a.shapes, a.verts, dt, clock, 0., 0);
    if (!grid_barrier(bar, status, a.barrier_polls)) return;
  }
}

// blocks of the persistent launch: every SM filled to its residency, no more
// than the work needs
template <typename R>
int persistent_blocks(const StepArgs<R>& a) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  cudaError_t e = a.has_convex
                      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_steps_kernel<R, true>,
                                                                      kPersistentThreads, 0)
                      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_steps_kernel<R, false>,
                                                                      kPersistentThreads, 0);
  if (e != cudaSuccess || per_sm < 1) return 0;
  const long long need = ((long long)a.n + kPersistentThreads - 1) / kPersistentThreads;
  return (int)std::max(1ll, std::min((long long)sms * per_sm, need));
}

template <typename R>
int launch_persistent_steps(const StepArgs<R>& a, cudaStream_t s, int n_steps, double dt, int gather_every,
                            int since_gather, int n_moving, double* clock, unsigned* bar, int* sums, int blocks) {
  if (n_steps <= 0 || a.n == 0) return 0;
  StepArgs<R> a0 = a;
  R dt_r = R(dt);
  void* args[] = {&a0, &n_steps, &dt_r, &dt, &gather_every, &since_gather, &n_moving, &clock, &bar, &sums};
  cudaError_t e = a.has_convex
                      ? cudaLaunchCooperativeKernel((const void*)persistent_steps_kernel<R, true>, dim3(blocks),
                                                    dim3(kPersistentThreads), args, 0, s)
                      : cudaLaunchCooperativeKernel((const void*)persistent_steps_kernel<R, false>, dim3(blocks),
                                                    dim3(kPersistentThreads), args, 0, s);
  return e == cudaSuccess ? 0 : GRAINS_GPU_CUDA_ERROR;
}

#define GG_INSTANTIATE(R)                                                                                  \
  template int launch_kick_move<R>(const StepArgs<R>&, cudaStream_t, int, double, int, double, double);    \
  template int launch_bin<R>(const StepArgs<R>&, cudaStream_t);                                            \
  template int launch_sort_and_gather<R>(const StepArgs<R>&, cudaStream_t, int, int);                      \
  template int launch_forces<R>(const StepArgs<R>&, cudaStream_t, double, int, int, int);                  \
  template int launch_zero_kdelta<R>(const StepArgs<R>&, cudaStream_t);                                    \
  template int launch_obstacle_force<R>(const StepArgs<R>&, double*, int, cudaStream_t);                    \
  template int launch_update_dynamic<R>(const StepArgs<R>&, cudaStream_t, const KinematicStage&);             \
  template int launch_set_fluid_ratio<R>(const StepArgs<R>&, cudaStream_t, const double*);                     \
  template int launch_set_velocities<R>(const StepArgs<R>&, cudaStream_t, const double*, const double*);      \
  template int launch_update_rows<R>(const StepArgs<R>&, cudaStream_t, const KinematicStage&, const long long*,  \
                                     long long, int*);                                                      \
  template int launch_pack_download<R>(const StepArgs<R>&, cudaStream_t, const DownloadStage&);              \
  template int launch_candidate_pairs<R>(const StepArgs<R>&, cudaStream_t, int, int, int*, int,           \
                                         unsigned long long*);                                            \
  template int persistent_blocks<R>(const StepArgs<R>&);                                                   \
  template int launch_persistent_steps<R>(const StepArgs<R>&, cudaStream_t, int, double, int, int, int, double*, \
                                          unsigned*, int*, int);

}  // namespace gg
