// adjoint.cuh -- differentiable run of the DEM step and its hand-written
// adjoint (no counterpart in the reference, which has no gradients).
//
// Scope: spheres with static box walls (the settling configurations), the
// Hooke and HookeMemory laws.  The run is the leapfrog of Grains::Simulation
// (Grains.cpp:169-174, 344-364) in upload order:
//
//   E_k:  (F_k, T_k, M_k) = Phi(X_k, V_k, W_k, M_{k-1}; theta)      k = 0..K
//         V_{k+1} = V_k + a_k F_k / m,  W_{k+1} = W_k + a_k T_k / I
//         X_{k+1} = X_k + dt V_{k+1}                                   k < K
//   a_0 = dt/2 (leapfrog start), a_k = dt (second half kick of step k plus
//   first half kick of step k+1), and after E_K the last half kick gives the
//   final velocities.  Phi is the force evaluation (27-cell broadphase, exact
//   double contact decisions, sphere-sphere and sphere-box closest points,
//   contact law, memory M of each contact), W the world angular velocity
//   (for spheres the body-frame RK3 of SecondOrderLeapFrog reduces to
//   W += a T / I), theta = (kn, en, muc, kt) of each contact law.  After E_0
//   the kdelta and rolling spring of every memory entry are zeroed, as the
//   leapfrog start of the reference does.
//
// Adjoint: lambda_X, lambda_V, lambda_W and the memory adjoint of each contact
// flow backwards through the same steps.  For each contact the kernel forms
// the vector-Jacobian product of its local map (relative position,
// velocities, angular velocities, memory in, theta) -> (force, the two
// torques, memory out) from forward-mode dual numbers (dual.cuh) run through
// the very contact-law templates of the step kernels, L input lanes per pass;
// per-particle sums are gathered in a fixed order (no atomics), so gradients
// are deterministic.  Checkpoints every S force evaluations hold the state and
// the contact rows; the reverse sweep recomputes one segment at a time.
//
// Data layout (N particles, C = contact slots per particle):
//   state slot:   X double4 (x, y, z, radius), V and W R4
//   contact rows: cnt[N]; other[C*N], link[C*N] (entry q of particle i at
//                 q*N + i, coalesced across a warp); memory out R[9][C*N]
//                 (kdelta, normal, rolling spring) of entries the particle
//                 owns (the lower index, or the particle for a wall).
//   other >= 0: particle index; other < 0: wall -(obstacle table index + 1).
//   link: owned entry -> its entry in the previous evaluation's rows (-1 new);
//         entry owned by the partner -> the partner's entry in these rows.
#pragma once

#include "common.cuh"
#include "contact_law.cuh"
#include "device_state.h"
#include "dual.cuh"
#include "sphere_contact.cuh"

namespace gg {

template <typename R>
struct AdjRows {
  int* cnt;
  int* other;
  int* link;
  R* mem;  // 9 components x cap*n
};

template <typename R>
struct AdjState {
  double4* X;
  typename Vec4<R>::type* V;
  typename Vec4<R>::type* W;
};

template <typename R>
struct AdjArgs {
  int n;
  int cap;       // contact slots per particle
  int n_cells;
  int n_laws;    // law table slots
  double dt;
  const SysDev* sys;
  const ShapeDev* shapes;
  const ObstacleDev* obs;
  const int* cell_obs_start;
  const int* cell_obs_idx;
  const LawParams<R>* laws;
  // static per particle, upload order
  const double4* md;     // mass, crust, equivalent radius, 0
  const int4* meta;      // id, material, shape, system
  const R* inertia;      // scalar moment of inertia (spheres)
  // grid scratch
  int* cell_count;
  int* cell_start;
  int* block_sums;
  int* perm;
  unsigned* key;
  unsigned* rank;
  int* status;
  unsigned long long* sig;  // [0] xor of a hash of every contact (evaluation, owner, partner, law
                            // branch flags), [1] count
};

// splitmix64 finaliser: hash of one contact entry for the run's signature
__device__ __forceinline__ unsigned long long contact_hash(int k, int i, int code, int branch) {
  unsigned long long z = ((unsigned long long)(unsigned)k << 40) ^ ((unsigned long long)(unsigned)i << 20) ^
                         (unsigned long long)(unsigned)code * 0x9E3779B97F4A7C15ull ^
                         (unsigned long long)(unsigned)branch << 61;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <typename R>
__device__ __forceinline__ typename Vec4<R>::type st3v(V3<R> a) {
  typename Vec4<R>::type r;
  r.x = a.x;
  r.y = a.y;
  r.z = a.z;
  r.w = R(0);
  return r;
}

// ---------------------------------------------------------------------------
// grid: counting sort of the particles of a state slot by cell
template <typename R>
__global__ void adj_bin_kernel(AdjArgs<R> a, const double4* X) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double4 x = X[i];
  const SysDev& S = a.sys[a.meta[i].w];
  int ci = int(floor(xdiv(xsub(x.x, S.ox), S.ex)));
  int cj = int(floor(xdiv(xsub(x.y, S.oy), S.ey)));
  int ck = int(floor(xdiv(xsub(x.z, S.oz), S.ez)));
  if (!(-1 < ci && ci < S.nbi && -1 < cj && cj < S.nbj && -1 < ck && ck < S.nbk)) {
    atomicOr(a.status, GRAINS_GPU_OUT_OF_GRID);
    ci = min(max(ci, 0), S.nbi - 1);
    cj = min(max(cj, 0), S.nbj - 1);
    ck = min(max(ck, 0), S.nbk - 1);
  }
  const unsigned key = (unsigned)(S.cell_offset + cj * S.nbk * S.nbi + ck * S.nbi + ci);
  a.key[i] = key;
  a.rank[i] = (unsigned)atomicAdd(&a.cell_count[key], 1);
}

constexpr int kAdjScanThreads = 1024;

__device__ __forceinline__ int adj_block_scan(int v, int* total) {
  __shared__ int ws[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    int s = lane < nw ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) ws[lane] = s;
  }
  __syncthreads();
  const int base = wid > 0 ? ws[wid - 1] : 0;
  *total = ws[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

// exclusive scan of cell_count into cell_start (C + 1 entries): per-block
// scans, one block over the block sums, then the add
static __global__ void __launch_bounds__(kAdjScanThreads) adj_scan_blocks(const int* in, int* out, int* sums, int n) {
  const int i = blockIdx.x * kAdjScanThreads + threadIdx.x;
  const int v = i < n ? in[i] : 0;
  int total;
  const int pre = adj_block_scan(v, &total);
  if (i < n) out[i] = pre;
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
static __global__ void __launch_bounds__(kAdjScanThreads) adj_scan_sums(int* sums, int nb, int* out, int n) {
  int run = 0;
  for (int base = 0; base < nb; base += kAdjScanThreads) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? sums[i] : 0;
    int total;
    const int pre = adj_block_scan(v, &total);
    if (i < nb) sums[i] = run + pre;
    run += total;
  }
  if (threadIdx.x == 0) out[n] = run;
}
static __global__ void adj_scan_add(int* out, const int* sums, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / kAdjScanThreads];
}

template <typename R>
__global__ void adj_scatter_kernel(AdjArgs<R> a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const long long slot = (long long)a.cell_start[a.key[i]] + a.rank[i];
  if (slot < 0 || slot >= a.n) {
    atomicOr(a.status, GRAINS_GPU_CUDA_ERROR);
    return;
  }
  a.perm[slot] = i;
}

// ---------------------------------------------------------------------------
// primal contact of one entry, seen from its owner (p0): the geometry in
// double exactly as in the step kernels, and the two bodies at the contact
template <typename R>
struct AdjContact {
  ContactGeom g;
  BodyAtContact<R> b0, b1;
  D3 A;       // owner centre
  D3 B;       // partner centre, or the wall's origin
  int wall;   // obstacle table index, -1 for a particle pair
  int law;    // law table slot
  double ra, rb;  // radii (rb unused for a wall)
};

template <typename R>
__device__ __forceinline__ bool adj_contact(const AdjArgs<R>& a, const AdjState<R>& st, int o, int code,
                                            AdjContact<R>& c) {
  const double4 xo = st.X[o];
  const double4 mo = a.md[o];
  const int4 meo = a.meta[o];
  const SysDev& S = a.sys[meo.w];
  c.A = d3(xo.x, xo.y, xo.z);
  c.ra = xo.w;
  c.rb = 0.;
  c.b0.v = v3<R>(st.V[o].x, st.V[o].y, st.V[o].z);
  c.b0.w = v3<R>(st.W[o].x, st.W[o].y, st.W[o].z);
  c.b0.mass = R(mo.x);
  c.b0.req = R(mo.z);
  if (code >= 0) {
    const int p = code;
    const double4 xp = st.X[p];
    const double4 mp = a.md[p];
    c.B = d3(xp.x, xp.y, xp.z);
    c.rb = xp.w;
    c.wall = -1;
    D3 ab;
    double nab;
    const double dist = sphere_sphere_overlap(c.A, xo.w, c.B, xp.w, &ab, &nab);
    if (!(dist < 0.)) return false;
    c.g = sphere_sphere_features(c.A, xo.w, ab, nab, dist, xadd(mo.y, mp.y));
    if (c.g.status) {
      atomicOr(a.status, GRAINS_GPU_CONTACT_ERROR);
      return false;
    }
    c.b1.v = v3<R>(st.V[p].x, st.V[p].y, st.V[p].z);
    c.b1.w = v3<R>(st.W[p].x, st.W[p].y, st.W[p].z);
    c.b1.mass = R(mp.x);
    c.b1.req = R(mp.z);
    c.law = S.law_offset + meo.y * S.n_mat + a.meta[p].y;
  } else {
    const int oidx = -code - 1;
    const ObstacleDev& O = a.obs[oidx];
    const ShapeDev& sh = a.shapes[O.shape];
    M3 ob;
    for (int t = 0; t < 9; ++t) ob.m[t] = O.b[t];
    c.B = d3(O.o[0], O.o[1], O.o[2]);
    c.wall = oidx;
    c.g = sphere_box(c.A, xo.w, xadd(mo.y, O.crust), ob, c.B, d3(sh.ext[0], sh.ext[1], sh.ext[2]));
    if (c.g.status) {
      atomicOr(a.status, GRAINS_GPU_CONTACT_ERROR);
      return false;
    }
    if (!(c.g.overlap < 0.)) return false;
    c.b1.v = v3<R>(R(O.vel[0]), R(O.vel[1]), R(O.vel[2]));
    c.b1.w = v3<R>(R(O.omega[0]), R(O.omega[1]), R(O.omega[2]));
    c.b1.mass = R(kObstacleMass);
    c.b1.req = R(pow((0.75 / kPi) * sh.volume, 1. / 3.));
    c.law = S.law_offset + meo.y * S.n_mat + O.material;
  }
  c.b0.lever = from_d3<R>(xsub3(c.g.point, c.A));
  c.b0.pos_minus_contact = from_d3<R>(xsub3(c.A, c.g.point));
  c.b1.lever = from_d3<R>(xsub3(c.g.point, c.B));
  c.b1.pos_minus_contact = from_d3<R>(xsub3(c.B, c.g.point));
  return true;
}

// memory entry of (owner o, partner code) in the previous evaluation's rows
template <typename R>
__device__ __forceinline__ int adj_find_memory(const AdjArgs<R>& a, const AdjRows<R>& prev, int o, int code,
                                               PairMemory<R>& m) {
  const int n = prev.cnt[o];
  const size_t cn = (size_t)a.cap * a.n;
  for (int q = 0; q < n; ++q) {
    const size_t r = (size_t)q * a.n + o;
    if (prev.other[r] == code) {
      m.kdelta = v3<R>(prev.mem[r], prev.mem[cn + r], prev.mem[2 * cn + r]);
      m.prev_normal = v3<R>(prev.mem[3 * cn + r], prev.mem[4 * cn + r], prev.mem[5 * cn + r]);
      m.spring = v3<R>(prev.mem[6 * cn + r], prev.mem[7 * cn + r], prev.mem[8 * cn + r]);
      return (int)r;
    }
  }
  return -1;
}

// contact entries of particle i: overlapping spheres of the 27 surrounding
// cells (sorted by index), then the walls linked to its cell (table order)
template <typename R>
__device__ int adj_collect(const AdjArgs<R>& a, const AdjState<R>& st, int i, int* list) {
  const double4 xi = st.X[i];
  const double4 mi = a.md[i];
  const SysDev& S = a.sys[a.meta[i].w];
  int ci = int(floor(xdiv(xsub(xi.x, S.ox), S.ex)));
  int cj = int(floor(xdiv(xsub(xi.y, S.oy), S.ey)));
  int ck = int(floor(xdiv(xsub(xi.z, S.oz), S.ez)));
  ci = min(max(ci, 0), S.nbi - 1);
  cj = min(max(cj, 0), S.nbj - 1);
  ck = min(max(ck, 0), S.nbk - 1);
  const D3 Xi = d3(xi.x, xi.y, xi.z);
  const int i0 = max(ci - 1, 0), i1 = min(ci + 1, S.nbi - 1);
  int cnt = 0;
  for (int dj = -1; dj <= 1; ++dj) {
    const int j = cj + dj;
    if (j < 0 || j >= S.nbj) continue;
    for (int dk = -1; dk <= 1; ++dk) {
      const int k = ck + dk;
      if (k < 0 || k >= S.nbk) continue;
      const int t0 = a.cell_start[S.cell_offset + j * S.nbk * S.nbi + k * S.nbi + i0];
      const int t1 = a.cell_start[S.cell_offset + j * S.nbk * S.nbi + k * S.nbi + i1 + 1];
      for (int t = t0; t < t1; ++t) {
        const int p = a.perm[t];
        if (p == i) continue;
        const double4 xp = st.X[p];
        D3 ab;
        double nab;
        if (!(sphere_sphere_overlap(Xi, xi.w, d3(xp.x, xp.y, xp.z), xp.w, &ab, &nab) < 0.)) continue;
        if (cnt < a.cap) {
          int u = cnt;
          while (u > 0 && list[u - 1] > p) {
            list[u] = list[u - 1];
            --u;
          }
          list[u] = p;
        }
        ++cnt;
      }
    }
  }
  const int cell = S.cell_offset + cj * S.nbk * S.nbi + ck * S.nbi + ci;
  for (int u = a.cell_obs_start[cell]; u < a.cell_obs_start[cell + 1]; ++u) {
    const int oidx = a.cell_obs_idx[u];
    const ObstacleDev& O = a.obs[oidx];
    if (!in_zone(d3(O.bbc[0], O.bbc[1], O.bbc[2]), d3(O.bbe[0], O.bbe[1], O.bbe[2]), Xi, xi.w, xi.w, xi.w)) continue;
    const ShapeDev& sh = a.shapes[O.shape];
    M3 ob;
    for (int t = 0; t < 9; ++t) ob.m[t] = O.b[t];
    const ContactGeom g = sphere_box(Xi, xi.w, xadd(mi.y, O.crust), ob, d3(O.o[0], O.o[1], O.o[2]),
                                     d3(sh.ext[0], sh.ext[1], sh.ext[2]));
    if (g.status) {
      atomicOr(a.status, GRAINS_GPU_CONTACT_ERROR);
      continue;
    }
    if (!(g.overlap < 0.)) continue;
    if (cnt < a.cap) list[cnt] = -oidx - 1;
    ++cnt;
  }
  if (cnt > a.cap) {
    atomicOr(a.status, GRAINS_GPU_HISTORY_FULL);
    cnt = a.cap;
  }
  return cnt;
}

template <typename R>
__device__ __forceinline__ LawResult<R> adj_law(const LawParams<R>& L, R dt, const AdjContact<R>& c, bool existed,
                                                PairMemory<R>& m, int* branch) {
  const V3<R> pen = from_d3<R>(c.g.overlap_vector);
  if (L.type == GRAINS_GPU_HOOKE_MEMORY) return hooke_memory(L, dt, pen, c.b0, c.b1, existed, m, branch);
  return hooke(L, pen, c.b0, c.b1, branch);
}

constexpr int kAdjMaxCap = 32;

// ---------------------------------------------------------------------------
// forward force evaluation E_k and the kick / drift that follows it, one
// thread per particle; writes the contact rows of E_k and the next state
template <typename R>
__global__ void __launch_bounds__(128) adj_eval_kernel(AdjArgs<R> a, AdjState<R> st, AdjRows<R> prev,
                                                       AdjRows<R> rows, AdjState<R> out, R h1, R h2, int drift,
                                                       int zero_memory, int k) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  int list[kAdjMaxCap];
  const int cnt = adj_collect(a, st, i, list);
  const double4 mdi = a.md[i];
  const SysDev& S = a.sys[a.meta[i].w];
  V3<R> F = v3<R>(R(S.gx * mdi.x), R(S.gy * mdi.x), R(S.gz * mdi.x));
  V3<R> T = v3<R>(R(0), R(0), R(0));
  const size_t cn = (size_t)a.cap * a.n;
  const R dt = R(a.dt);
  for (int q = 0; q < cnt; ++q) {
    const int code = list[q];
    const bool own = code < 0 || i < code;
    const int o = own ? i : code;
    const int pcode = own ? code : i;
    const size_t r = (size_t)q * a.n + i;
    rows.other[r] = code;
    AdjContact<R> c;
    if (!adj_contact(a, st, o, pcode, c)) {
      rows.link[r] = -1;
      continue;
    }
    const LawParams<R> L = a.laws[c.law];
    PairMemory<R> m;
    m.kdelta = m.prev_normal = m.spring = v3<R>(R(0), R(0), R(0));
    const int pr = L.type == GRAINS_GPU_HOOKE_MEMORY ? adj_find_memory(a, prev, o, pcode, m) : -1;
    int branch = 0;
    const LawResult<R> res = adj_law(L, dt, c, pr >= 0, m, &branch);
    const V3<R> f = own ? res.force : -res.force;
    F = F + f;
    T = T + cross(own ? c.b0.lever : c.b1.lever, f);
    if (L.rolling || L.kr != R(0)) T = T + (own ? res.torque : -res.torque);
    if (own) {
      atomicXor(&a.sig[0], contact_hash(k, i, code, branch));
      atomicAdd(&a.sig[1], 1ull);
      rows.link[r] = pr;
      if (zero_memory) m.kdelta = m.spring = v3<R>(R(0), R(0), R(0));
      rows.mem[r] = m.kdelta.x;
      rows.mem[cn + r] = m.kdelta.y;
      rows.mem[2 * cn + r] = m.kdelta.z;
      rows.mem[3 * cn + r] = m.prev_normal.x;
      rows.mem[4 * cn + r] = m.prev_normal.y;
      rows.mem[5 * cn + r] = m.prev_normal.z;
      rows.mem[6 * cn + r] = m.spring.x;
      rows.mem[7 * cn + r] = m.spring.y;
      rows.mem[8 * cn + r] = m.spring.z;
    } else {
      rows.link[r] = -2;  // resolved by adj_link_kernel
    }
  }
  rows.cnt[i] = cnt;
  // kick(s), drift
  const R mass = R(mdi.x);
  const R I = a.inertia[i];
  const V3<R> acc = dv(F, mass * R(1));
  const V3<R> alpha = dv(T, R(1) * I);
  V3<R> v = v3<R>(st.V[i].x, st.V[i].y, st.V[i].z);
  V3<R> w = v3<R>(st.W[i].x, st.W[i].y, st.W[i].z);
  v = v + sc(acc, h1);
  w = w + sc(alpha, h1);
  if (h2 != R(0)) {
    v = v + sc(acc, h2);
    w = w + sc(alpha, h2);
  }
  double4 x = st.X[i];
  if (drift) {
    const V3<double> tm = sc(v3<double>(double(v.x), double(v.y), double(v.z)), a.dt);
    x.x = x.x + tm.x;
    x.y = x.y + tm.y;
    x.z = x.z + tm.z;
    if (norm(tm) > mdi.y) atomicOr(a.status, GRAINS_GPU_MOTION_ERROR);
  }
  out.X[i] = x;
  out.V[i] = st3v<R>(v);
  out.W[i] = st3v<R>(w);
}

// entries owned by the partner: the partner's entry index in the same rows
template <typename R>
__global__ void adj_link_kernel(AdjArgs<R> a, AdjRows<R> rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int cnt = rows.cnt[i];
  for (int q = 0; q < cnt; ++q) {
    const size_t r = (size_t)q * a.n + i;
    if (rows.link[r] != -2) continue;
    const int p = rows.other[r];
    int found = -1;
    const int np = rows.cnt[p];
    for (int u = 0; u < np; ++u)
      if (rows.other[(size_t)u * a.n + p] == i) found = u * a.n + p;
    rows.link[r] = found;
  }
}


// ---------------------------------------------------------------------------
// reverse sweep

// inputs of one contact's local map, in this order:
//   0-2 relative position (pair: partner - owner; wall: particle - wall origin)
//   3-5 owner velocity, 6-8 partner velocity, 9-11 owner angular velocity,
//   12-14 partner angular velocity, 15-17 kdelta in, 18-20 normal in,
//   21-23 rolling spring in, 24 kn, 25 en, 26 muc, 27 kt
constexpr int kAdjInputs = 28;

template <typename T, int L>
__device__ __forceinline__ void set_value(V3<Dual<T, L>>& x, V3<T> v) {
  x.x.v = v.x;
  x.y.v = v.y;
  x.z.v = v.z;
}

// Box-frame region of a sphere centre (the branches of Box::
// IntersectionPointSPHERE, Box.cpp:466-718): s[a] = +1 / -1 beyond the + / -
// face of axis a, 0 between the two faces
__device__ __forceinline__ void box_region(D3 e, D3 c, int s[3]) {
  s[0] = c.x > e.x ? 1 : (c.x < -e.x ? -1 : 0);
  s[1] = c.y > e.y ? 1 : (c.y < -e.y ? -1 : 0);
  s[2] = c.z > e.z ? 1 : (c.z < -e.z ? -1 : 0);
}

template <typename T, int L>
__device__ __forceinline__ Dual<T, L>& comp(V3<Dual<T, L>>& v, int a) {
  return a == 0 ? v.x : (a == 1 ? v.y : v.z);
}

// One pass of L forward-mode lanes over the contact's local map.  The lanes
// carry inputs act[base .. base + L); grad[m] receives the vector-Jacobian
// product <lam, d outputs / d input m> for each of them.  The geometry is
// rebuilt in dual arithmetic (its values then replaced by the exact double
// ones of the step), the law is the step kernels' own template.
template <typename R, int L>
__device__ void adj_contact_vjp_pass(const AdjArgs<R>& a, const AdjContact<R>& c, const LawParams<R>& L0,
                                     bool existed, const R in[kAdjInputs], const int* act, int n_act, int base,
                                     const V3<R> lam[6], R grad[kAdjInputs]) {
  using D = Dual<R, L>;
  auto mk = [&](int m) -> D {
    int lane = -1;
#pragma unroll
    for (int l = 0; l < L; ++l)
      if (base + l < n_act && act[base + l] == m) lane = l;
    return seeded<R, L>(in[m], lane);
  };
  auto mk3 = [&](int m) -> V3<D> { return V3<D>{mk(m), mk(m + 1), mk(m + 2)}; };
  auto cst3 = [](V3<R> v) -> V3<D> { return V3<D>{D(v.x), D(v.y), D(v.z)}; };
  const bool wall = c.wall >= 0;
  V3<D> lev0, lev1, pen;
  if (!wall) {
    // ClosestPointSPHERESPHERE (RigidBodyWithCrust.cpp:611-638) as a function of B - A
    const V3<D> ab = mk3(0);
    const D nab = norm(ab);
    const D dist = nab - D(xadd(c.ra, c.rb));
    const D s = D(c.ra) + D(0.5) * dist;
    lev0 = dv(sc(ab, s), nab);
    pen = sc(dv(ab, nab), dist);
    lev1 = lev0 - ab;
  } else {
    // ClosestPointSPHEREBOX (RigidBodyWithCrust.cpp:647-721) as a function of
    // the centre relative to the wall origin, in the region of the step
    const ObstacleDev& O = a.obs[c.wall];
    const ShapeDev& sh = a.shapes[O.shape];
    const D3 e = d3(sh.ext[0], sh.ext[1], sh.ext[2]);
    M3 ob;
    for (int t = 0; t < 9; ++t) ob.m[t] = O.b[t];
    const M3 bt = mtranspose(ob);
    const D3 io = d3(-xdot(mrow(bt, 0), c.B), -xdot(mrow(bt, 1), c.B), -xdot(mrow(bt, 2), c.B));
    const D3 lc = xapply(bt, io, c.A);
    int sr[3];
    box_region(e, lc, sr);
    const V3<D> rel = mk3(0);
    V3<D> loc;
    loc.x = D(R(ob.m[0])) * rel.x + D(R(ob.m[3])) * rel.y + D(R(ob.m[6])) * rel.z;
    loc.y = D(R(ob.m[1])) * rel.x + D(R(ob.m[4])) * rel.y + D(R(ob.m[7])) * rel.z;
    loc.z = D(R(ob.m[2])) * rel.x + D(R(ob.m[5])) * rel.y + D(R(ob.m[8])) * rel.z;
    const R ev[3] = {R(e.x), R(e.y), R(e.z)};
    const int nz = (sr[0] != 0) + (sr[1] != 0) + (sr[2] != 0);
    V3<D> cp = loc;
    D ov;
    if (nz == 1) {
      const int ax = sr[0] != 0 ? 0 : (sr[1] != 0 ? 1 : 2);
      const D g = comp(loc, ax);
      const D nd = sr[ax] > 0 ? g - D(ev[ax]) : D(-ev[ax]) - g;
      ov = nd - D(c.ra);
      comp(cp, ax) = sr[ax] > 0 ? D(ev[ax]) + D(0.5) * ov : D(-ev[ax]) - D(0.5) * ov;
    } else {
      V3<D> d;
      d.x = sr[0] != 0 ? loc.x - D(R(sr[0]) * ev[0]) : D(0.);
      d.y = sr[1] != 0 ? loc.y - D(R(sr[1]) * ev[1]) : D(0.);
      d.z = sr[2] != 0 ? loc.z - D(R(sr[2]) * ev[2]) : D(0.);
      const D nd = norm(d);
      ov = nd - D(c.ra);
      cp = loc - sc(d, D(1.) + D(0.5) * ov / nd);
    }
    V3<D> prel;
    prel.x = D(R(ob.m[0])) * cp.x + D(R(ob.m[1])) * cp.y + D(R(ob.m[2])) * cp.z;
    prel.y = D(R(ob.m[3])) * cp.x + D(R(ob.m[4])) * cp.y + D(R(ob.m[5])) * cp.z;
    prel.z = D(R(ob.m[6])) * cp.x + D(R(ob.m[7])) * cp.y + D(R(ob.m[8])) * cp.z;
    lev0 = prel - rel;
    pen = sc(lev0, ov / norm(lev0));
    lev1 = prel;
  }
  set_value(lev0, c.b0.lever);
  set_value(lev1, c.b1.lever);
  set_value(pen, from_d3<R>(c.g.overlap_vector));
  BodyAtContact<D> b0, b1;
  b0.v = mk3(3);
  b0.w = mk3(9);
  b0.lever = lev0;
  b0.pos_minus_contact = -lev0;
  set_value(b0.pos_minus_contact, c.b0.pos_minus_contact);
  b0.mass = D(c.b0.mass);
  b0.req = D(c.b0.req);
  b1.v = wall ? cst3(c.b1.v) : mk3(6);
  b1.w = wall ? cst3(c.b1.w) : mk3(12);
  b1.lever = lev1;
  b1.pos_minus_contact = -lev1;
  set_value(b1.pos_minus_contact, c.b1.pos_minus_contact);
  b1.mass = D(c.b1.mass);
  b1.req = D(c.b1.req);
  LawParams<D> Ld;
  Ld.type = L0.type;
  Ld.rolling = L0.rolling;
  Ld.kn = mk(24);
  Ld.en = mk(25);
  Ld.muc = mk(26);
  Ld.kt = mk(27);
  Ld.etat = D(L0.etat);
  Ld.mur = D(L0.mur);
  Ld.etarpf = D(L0.etarpf);
  Ld.epst = D(L0.epst);
  Ld.kr = D(L0.kr);
  // beta = ln(en) / sqrt(pi^2 + ln^2 en): d beta / d en = pi^2 / (en (pi^2 + ln^2 en)^1.5)
  Ld.beta = D(L0.beta);
  {
    const double en = double(L0.en), u = log(en);
    const R dbde = R(kPi * kPi / (en * pow(kPi * kPi + u * u, 1.5)));
#pragma unroll
    for (int l = 0; l < L; ++l) Ld.beta.d[l] = dbde * Ld.en.d[l];
  }
  PairMemory<D> m;
  m.kdelta = mk3(15);
  m.prev_normal = mk3(18);
  m.spring = mk3(21);
  const LawResult<D> res = L0.type == GRAINS_GPU_HOOKE_MEMORY
                               ? hooke_memory(Ld, D(R(a.dt)), pen, b0, b1, existed, m)
                               : hooke(Ld, pen, b0, b1);
  const V3<D> f = res.force;
  V3<D> Ti = cross(lev0, f);
  V3<D> Tj = cross(lev1, -f);
  if (L0.rolling || L0.kr != R(0)) {
    Ti = Ti + res.torque;
    Tj = Tj - res.torque;
  }
  R acc[L];
#pragma unroll
  for (int l = 0; l < L; ++l) acc[l] = R(0);
  accumulate_vjp(f, lam[0], acc);
  accumulate_vjp(Ti, lam[1], acc);
  accumulate_vjp(Tj, lam[2], acc);
  accumulate_vjp(m.kdelta, lam[3], acc);
  accumulate_vjp(m.prev_normal, lam[4], acc);
  accumulate_vjp(m.spring, lam[5], acc);
#pragma unroll
  for (int l = 0; l < L; ++l)
    if (base + l < n_act) grad[act[base + l]] = acc[l];
}

// RA: adjoint of every contact of evaluation E_k, one thread per particle
// over the entries it owns.  lamF / lamT: adjoints of the particles' force and
// torque sums of E_k; lam_out: adjoints of the memory written by E_k (null at
// the last evaluation); lam_in (zeroed before): receives the adjoints of the
// memory E_k read, at the previous rows' entry; radj: per owned entry the
// adjoints of the relative position (3), the two velocities and the two
// angular velocities (12); gtheta[(law * n + i) * 4 + .] accumulates the
// parameter adjoints of the particle's owned contacts.
template <typename R, int L>
__global__ void __launch_bounds__(128) adj_reverse_contacts_kernel(AdjArgs<R> a, AdjState<R> st, AdjRows<R> prev,
                                                                   AdjRows<R> rows,
                                                                   const typename Vec4<R>::type* lamF,
                                                                   const typename Vec4<R>::type* lamT,
                                                                   const R* lam_out, R* lam_in, R* radj,
                                                                   double* gtheta, int zero_memory_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const size_t cn = (size_t)a.cap * a.n;
  const int cnt = rows.cnt[i];
  for (int q = 0; q < cnt; ++q) {
    const size_t r = (size_t)q * a.n + i;
    const int code = rows.other[r];
    if (!(code < 0 || i < code)) continue;
    AdjContact<R> c;
    R grad[kAdjInputs];
#pragma unroll
    for (int m = 0; m < kAdjInputs; ++m) grad[m] = R(0);
    if (adj_contact(a, st, i, code, c)) {
      const LawParams<R> L0 = a.laws[c.law];
      const bool memlaw = L0.type == GRAINS_GPU_HOOKE_MEMORY;
      const int pr = memlaw ? rows.link[r] : -1;
      const bool existed = pr >= 0;
      R in[kAdjInputs];
      const D3 rel = xsub3(c.wall >= 0 ? c.A : c.B, c.wall >= 0 ? c.B : c.A);
      in[0] = R(rel.x);
      in[1] = R(rel.y);
      in[2] = R(rel.z);
      in[3] = c.b0.v.x; in[4] = c.b0.v.y; in[5] = c.b0.v.z;
      in[6] = c.b1.v.x; in[7] = c.b1.v.y; in[8] = c.b1.v.z;
      in[9] = c.b0.w.x; in[10] = c.b0.w.y; in[11] = c.b0.w.z;
      in[12] = c.b1.w.x; in[13] = c.b1.w.y; in[14] = c.b1.w.z;
      for (int t = 0; t < 9; ++t) in[15 + t] = existed ? prev.mem[t * cn + pr] : R(0);
      in[24] = L0.kn;
      in[25] = L0.en;
      in[26] = L0.muc;
      in[27] = L0.kt;
      int act[kAdjInputs];
      int n_act = 0;
      for (int m = 0; m < 6; ++m) act[n_act++] = m;
      if (c.wall < 0)
        for (int m = 6; m < 9; ++m) act[n_act++] = m;
      for (int m = 9; m < 12; ++m) act[n_act++] = m;
      if (c.wall < 0)
        for (int m = 12; m < 15; ++m) act[n_act++] = m;
      if (existed)
        for (int m = 15; m < 21; ++m) act[n_act++] = m;
      if (existed && L0.rolling)
        for (int m = 21; m < 24; ++m) act[n_act++] = m;
      act[n_act++] = 24;
      act[n_act++] = 25;
      act[n_act++] = 26;
      if (memlaw) act[n_act++] = 27;
      V3<R> lam[6];
      const typename Vec4<R>::type fi = lamF[i], ti = lamT[i];
      lam[0] = v3<R>(fi.x, fi.y, fi.z);
      lam[1] = v3<R>(ti.x, ti.y, ti.z);
      lam[2] = v3<R>(R(0), R(0), R(0));
      if (c.wall < 0) {
        const typename Vec4<R>::type fj = lamF[code], tj = lamT[code];
        lam[0] = lam[0] - v3<R>(fj.x, fj.y, fj.z);
        lam[2] = v3<R>(tj.x, tj.y, tj.z);
      }
      for (int t = 0; t < 3; ++t) lam[3 + t] = v3<R>(R(0), R(0), R(0));
      if (lam_out && memlaw) {
        lam[3] = v3<R>(lam_out[r], lam_out[cn + r], lam_out[2 * cn + r]);
        lam[4] = v3<R>(lam_out[3 * cn + r], lam_out[4 * cn + r], lam_out[5 * cn + r]);
        lam[5] = v3<R>(lam_out[6 * cn + r], lam_out[7 * cn + r], lam_out[8 * cn + r]);
      }
      if (zero_memory_out) lam[3] = lam[5] = v3<R>(R(0), R(0), R(0));
      for (int base = 0; base < n_act; base += L)
        adj_contact_vjp_pass<R, L>(a, c, L0, existed, in, act, n_act, base, lam, grad);
      if (existed)
        for (int t = 0; t < 9; ++t) lam_in[t * cn + pr] = grad[15 + t];
      double* g = gtheta + ((size_t)c.law * a.n + i) * 4;
      g[0] += double(grad[24]);
      g[1] += double(grad[25]);
      g[2] += double(grad[26]);
      g[3] += double(grad[27]);
    }
    for (int t = 0; t < 15; ++t) radj[t * cn + r] = grad[t];
  }
}

// RB: per-particle sums of the contact adjoints of E_k in row order, the
// adjoints of X_k, V_k, W_k; then the kick and drift that produced them:
// lamF_{k-1} = a_{k-1} / m (lamV_k + dt lamX_k), lamT_{k-1} = a_{k-1} / I lamW_k.
// At k = 0 (coef_prev = 0) the adjoints of the initial state are written out.
template <typename R>
__global__ void adj_reverse_particles_kernel(AdjArgs<R> a, AdjRows<R> rows, const R* radj,
                                             typename Vec4<R>::type* aX, typename Vec4<R>::type* aV,
                                             typename Vec4<R>::type* aW, typename Vec4<R>::type* aF,
                                             typename Vec4<R>::type* aT, double coef_prev, double* gX,
                                             double* gV, double* gW) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const size_t cn = (size_t)a.cap * a.n;
  V3<R> sx = v3<R>(aX[i].x, aX[i].y, aX[i].z);
  V3<R> sv = v3<R>(aV[i].x, aV[i].y, aV[i].z);
  V3<R> sw = v3<R>(aW[i].x, aW[i].y, aW[i].z);
  const int cnt = rows.cnt[i];
  for (int q = 0; q < cnt; ++q) {
    const size_t r = (size_t)q * a.n + i;
    const int code = rows.other[r];
    const V3<R> gr = v3<R>(radj[r], radj[cn + r], radj[2 * cn + r]);
    if (code < 0) {  // wall: relative position = X_i - origin
      sx = sx + gr;
      sv = sv + v3<R>(radj[3 * cn + r], radj[4 * cn + r], radj[5 * cn + r]);
      sw = sw + v3<R>(radj[9 * cn + r], radj[10 * cn + r], radj[11 * cn + r]);
    } else if (i < code) {  // owner: relative position = X_partner - X_i
      sx = sx - gr;
      sv = sv + v3<R>(radj[3 * cn + r], radj[4 * cn + r], radj[5 * cn + r]);
      sw = sw + v3<R>(radj[9 * cn + r], radj[10 * cn + r], radj[11 * cn + r]);
    } else {  // partner's entry
      const int lk = rows.link[r];
      if (lk < 0) continue;
      const size_t o = (size_t)lk;
      sx = sx + v3<R>(radj[o], radj[cn + o], radj[2 * cn + o]);
      sv = sv + v3<R>(radj[6 * cn + o], radj[7 * cn + o], radj[8 * cn + o]);
      sw = sw + v3<R>(radj[12 * cn + o], radj[13 * cn + o], radj[14 * cn + o]);
    }
  }
  if (coef_prev > 0.) {
    const V3<R> vv = sv + sc(sx, R(a.dt));
    const R m = R(a.md[i].x);
    const R I = a.inertia[i];
    aF[i] = st3v<R>(sc(vv, R(coef_prev) / m));
    aT[i] = st3v<R>(sc(sw, R(coef_prev) / I));
    aX[i] = st3v<R>(sx);
    aV[i] = st3v<R>(vv);
    aW[i] = st3v<R>(sw);
  } else {
    gX[3 * i] = double(sx.x);
    gX[3 * i + 1] = double(sx.y);
    gX[3 * i + 2] = double(sx.z);
    gV[3 * i] = double(sv.x);
    gV[3 * i + 1] = double(sv.y);
    gV[3 * i + 2] = double(sv.z);
    gW[3 * i] = double(sw.x);
    gW[3 * i + 1] = double(sw.y);
    gW[3 * i + 2] = double(sw.z);
  }
}

// adjoint at the end of the run from dL/d(final position, velocity, angular
// velocity): v_fin = V_K + dt/2 F_K / m, w_fin = W_K + dt/2 T_K / I, x_fin = X_K
template <typename R>
__global__ void adj_init_kernel(AdjArgs<R> a, const double* gx, const double* gv, const double* gw,
                                typename Vec4<R>::type* aX, typename Vec4<R>::type* aV,
                                typename Vec4<R>::type* aW, typename Vec4<R>::type* aF,
                                typename Vec4<R>::type* aT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const V3<R> x = v3<R>(R(gx[3 * i]), R(gx[3 * i + 1]), R(gx[3 * i + 2]));
  const V3<R> v = v3<R>(R(gv[3 * i]), R(gv[3 * i + 1]), R(gv[3 * i + 2]));
  const V3<R> w = v3<R>(R(gw[3 * i]), R(gw[3 * i + 1]), R(gw[3 * i + 2]));
  const R h = R(0.5 * a.dt);
  aX[i] = st3v<R>(x);
  aV[i] = st3v<R>(v);
  aW[i] = st3v<R>(w);
  aF[i] = st3v<R>(sc(v, h / R(a.md[i].x)));
  aT[i] = st3v<R>(sc(w, h / a.inertia[i]));
}

// the parameter adjoints summed over particles in a fixed order: one block
// per (law slot, parameter)
static __global__ void adj_reduce_theta_kernel(const double* gtheta, int n, double* out) {
  __shared__ double sh[256];
  const int slot = blockIdx.x / 4, p = blockIdx.x % 4;
  double s = 0.;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += gtheta[((size_t)slot * n + i) * 4 + p];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// initial state and static data of the context, into upload order
template <typename R>
__global__ void adj_gather_kernel(int n, const double4* xr, const double4* md, const int4* meta, const int* orig,
                                  const typename Vec4<R>::type* v, const typename Vec4<R>::type* w,
                                  const typename Vec4<R>::type* inertia, double4* X, typename Vec4<R>::type* V,
                                  typename Vec4<R>::type* W, double4* md_u, int4* meta_u, R* inertia_u) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int i = orig[s];
  if (i < 0 || i >= n) return;
  X[i] = xr[s];
  V[i] = v[s];
  W[i] = w[s];
  md_u[i] = md[s];
  meta_u[i] = meta[s];
  inertia_u[i] = inertia[s].x;
}

}  // namespace gg

// ---------------------------------------------------------------------------
// host side: the engine of one precision
#include <algorithm>
#include <vector>

#include "adjoint.h"

namespace gg {

template <typename R, int LANES>
class AdjEngineT : public AdjointEngine {
  using R4 = typename Vec4<R>::type;

 public:
  AdjEngineT(const ContextView& v, int checkpoint_every) {
    n_ = v.n;
    cap_ = std::min(std::max(v.hist_cap, 1), kAdjMaxCap);
    S_ = std::max(checkpoint_every, 1);
    n_cells_ = v.n_cells;
    n_laws_ = v.n_laws;
    stream_ = v.stream;
    const size_t N = (size_t)n_, cn = (size_t)cap_ * n_;
    ok_ = true;
    md_ = alloc<double4>(N);
    meta_ = alloc<int4>(N);
    inertia_ = alloc<R>(N);
    cell_count_ = alloc<int>(n_cells_);
    cell_start_ = alloc<int>((size_t)n_cells_ + 1);
    block_sums_ = alloc<int>((size_t)n_cells_ / kAdjScanThreads + 2);
    perm_ = alloc<int>(N);
    key_ = alloc<unsigned>(N);
    rank_ = alloc<unsigned>(N);
    status_ = alloc<int>(1);
    sig_ = alloc<unsigned long long>(4);
    tX_ = alloc<double4>((S_ + 1) * N);
    tV_ = alloc<R4>((S_ + 1) * N);
    tW_ = alloc<R4>((S_ + 1) * N);
    tcnt_ = alloc<int>((S_ + 1) * N);
    tother_ = alloc<int>((S_ + 1) * cn);
    tlink_ = alloc<int>((S_ + 1) * cn);
    tmem_ = alloc<R>((S_ + 1) * 9 * cn);
    lam_[0] = alloc<R>(9 * cn);
    lam_[1] = alloc<R>(9 * cn);
    radj_ = alloc<R>(15 * cn);
    aX_ = alloc<R4>(N);
    aV_ = alloc<R4>(N);
    aW_ = alloc<R4>(N);
    aF_ = alloc<R4>(N);
    aT_ = alloc<R4>(N);
    gtheta_ = alloc<double>((size_t)n_laws_ * N * 4);
    theta_ = alloc<double>((size_t)n_laws_ * 4);
    gin_ = alloc<double>(9 * N);
    gout_ = alloc<double>(9 * N);
  }
  ~AdjEngineT() override {
    for (void* p : pool_) cudaFree(p);
    for (void* p : ck_pool_) cudaFree(p);
  }
  bool ok() const { return ok_; }
  int n_law_slots() const override { return n_laws_; }
  size_t device_bytes() const override { return bytes_; }

  int forward(const ContextView& v, int K, double dt, double* x, double* vel, double* w, std::string& err) override {
    if (v.n != n_ || v.n_cells != n_cells_ || v.n_laws != n_laws_) {
      err = "the context changed size since the adjoint was created";
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
    if (!v.spheres_only || !v.box_walls_only || v.n_moving) {
      err = "the differentiable run supports spheres with static box walls only";
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
    if (!v.hooke_laws_only) {
      err = "the differentiable run supports the Hooke and HookeMemory laws only";
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
    if (K < 0 || !(dt > 0.)) {
      err = "n_steps must be >= 0 and dt > 0";
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
    view_ = v;
    K_ = K;
    dt_ = dt;
    n_seg_ = (K + 1 + S_ - 1) / S_;
    if (int rc = alloc_checkpoints(err)) return rc;
    const int g = grid(n_);
    adj_gather_kernel<R><<<g, 256, 0, stream_>>>(n_, v.xr, v.md, v.meta, v.orig, (const R4*)v.v, (const R4*)v.w,
                                                 (const R4*)v.inertia, tX_, tV_, tW_, md_, meta_, inertia_);
    if (cudaMemsetAsync(tcnt_, 0, (size_t)n_ * sizeof(int), stream_) != cudaSuccess ||
        cudaMemsetAsync(sig_, 0, 4 * sizeof(unsigned long long), stream_) != cudaSuccess ||
        cudaMemsetAsync(status_, 0, sizeof(int), stream_) != cudaSuccess)
      return cuda_err(err);
    for (int j = 0; j < n_seg_; ++j) {
      const int k0 = j * S_, len = std::min(S_, K + 1 - k0);
      if (int rc = save_checkpoint(j)) return cuda_err(err, rc);
      for (int t = 0; t < len; ++t)
        if (int rc = eval(k0 + t, t, false)) return cuda_err(err, rc);
      if (j + 1 < n_seg_)
        if (int rc = shift_slot(len)) return cuda_err(err, rc);
      last_len_ = len;
    }
    // final state: slot last_len_ of the last segment
    std::vector<double4> hx(n_);
    std::vector<R4> hv(n_), hw(n_);
    const size_t off = (size_t)last_len_ * n_;
    if (cudaMemcpyAsync(hx.data(), tX_ + off, n_ * sizeof(double4), cudaMemcpyDeviceToHost, stream_) ||
        cudaMemcpyAsync(hv.data(), tV_ + off, n_ * sizeof(R4), cudaMemcpyDeviceToHost, stream_) ||
        cudaMemcpyAsync(hw.data(), tW_ + off, n_ * sizeof(R4), cudaMemcpyDeviceToHost, stream_))
      return cuda_err(err);
    if (int rc = check_status(err)) return rc;
    for (int i = 0; i < n_; ++i) {
      if (x) {
        x[3 * i] = hx[i].x;
        x[3 * i + 1] = hx[i].y;
        x[3 * i + 2] = hx[i].z;
      }
      if (vel) {
        vel[3 * i] = double(hv[i].x);
        vel[3 * i + 1] = double(hv[i].y);
        vel[3 * i + 2] = double(hv[i].z);
      }
      if (w) {
        w[3 * i] = double(hw[i].x);
        w[3 * i + 1] = double(hw[i].y);
        w[3 * i + 2] = double(hw[i].z);
      }
    }
    if (cudaMemcpy(sig_host_, sig_, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
      return cuda_err(err);
    have_forward_ = true;
    return 0;
  }
  void signature(unsigned long long* sig, long long* n_contacts) const override {
    *sig = sig_host_[0];
    *n_contacts = (long long)sig_host_[1];
  }

  int backward(const double* gx, const double* gv, const double* gw, double* ox, double* ov, double* ow,
               double* glaw, int n_glaw, std::string& err) override {
    if (!have_forward_) {
      err = "backward needs a forward run first";
      return GRAINS_GPU_NOT_READY;
    }
    const size_t N = (size_t)n_, cn = (size_t)cap_ * n_;
    std::vector<double> hin(9 * N, 0.);
    for (size_t k = 0; k < 3 * N; ++k) {
      hin[k] = gx ? gx[k] : 0.;
      hin[3 * N + k] = gv ? gv[k] : 0.;
      hin[6 * N + k] = gw ? gw[k] : 0.;
    }
    if (cudaMemcpyAsync(gin_, hin.data(), 9 * N * sizeof(double), cudaMemcpyHostToDevice, stream_) != cudaSuccess)
      return cuda_err(err);
    AdjArgs<R> a = args();
    const int g = grid(n_);
    adj_init_kernel<R><<<g, 256, 0, stream_>>>(a, gin_, gin_ + 3 * N, gin_ + 6 * N, aX_, aV_, aW_, aF_, aT_);
    if (cudaMemsetAsync(gtheta_, 0, (size_t)n_laws_ * N * 4 * sizeof(double), stream_) != cudaSuccess ||
        cudaMemsetAsync(lam_[0], 0, 9 * cn * sizeof(R), stream_) != cudaSuccess ||
        cudaMemsetAsync(status_, 0, sizeof(int), stream_) != cudaSuccess)
      return cuda_err(err);
    int cur = 0;
    for (int j = n_seg_ - 1; j >= 0; --j) {
      const int k0 = j * S_, len = std::min(S_, K_ + 1 - k0);
      if (int rc = restore_checkpoint(j)) return cuda_err(err, rc);
      for (int t = 0; t < len; ++t)
        if (int rc = eval(k0 + t, t, true)) return cuda_err(err, rc);
      for (int t = len - 1; t >= 0; --t) {
        const int k = k0 + t;
        const int nxt = 1 - cur;
        if (cudaMemsetAsync(lam_[nxt], 0, 9 * cn * sizeof(R), stream_) != cudaSuccess) return cuda_err(err);
        adj_reverse_contacts_kernel<R, LANES><<<grid(n_, 128), 128, 0, stream_>>>(
            a, state(t), rows(t), rows(t + 1), aF_, aT_, lam_[cur], lam_[nxt], radj_, gtheta_, k == 0 ? 1 : 0);
        const double coef_prev = k == 0 ? 0. : (k - 1 == 0 ? 0.5 * dt_ : dt_);
        adj_reverse_particles_kernel<R><<<g, 256, 0, stream_>>>(a, rows(t + 1), radj_, aX_, aV_, aW_, aF_, aT_,
                                                                coef_prev, gout_, gout_ + 3 * N, gout_ + 6 * N);
        if (cudaGetLastError() != cudaSuccess) return cuda_err(err);
        cur = nxt;
      }
    }
    adj_reduce_theta_kernel<<<n_laws_ * 4, 256, 0, stream_>>>(gtheta_, n_, theta_);
    std::vector<double> hout(9 * N), hth((size_t)n_laws_ * 4);
    if (cudaMemcpyAsync(hout.data(), gout_, 9 * N * sizeof(double), cudaMemcpyDeviceToHost, stream_) ||
        cudaMemcpyAsync(hth.data(), theta_, hth.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_))
      return cuda_err(err);
    if (int rc = check_status(err)) return rc;
    for (size_t k = 0; k < 3 * N; ++k) {
      if (ox) ox[k] = hout[k];
      if (ov) ov[k] = hout[3 * N + k];
      if (ow) ow[k] = hout[6 * N + k];
    }
    if (glaw)
      for (int k = 0; k < n_glaw && k < 4 * n_laws_; ++k) glaw[k] = hth[k];
    return 0;
  }

 private:
  template <typename T>
  T* alloc(size_t count) {
    void* p = nullptr;
    const size_t b = std::max<size_t>(count, 1) * sizeof(T);
    if (cudaMalloc(&p, b) != cudaSuccess) {
      ok_ = false;
      return nullptr;
    }
    bytes_ += b;
    pool_.push_back(p);
    return static_cast<T*>(p);
  }
  static int grid(long long n, int block = 256) { return (int)((n + block - 1) / block); }
  int cuda_err(std::string& err, int rc = GRAINS_GPU_CUDA_ERROR) {
    cudaError_t e = cudaGetLastError();
    err = std::string("adjoint: CUDA error ") + cudaGetErrorString(e);
    return rc;
  }
  int check_status(std::string& err) {
    int st = 0;
    if (cudaMemcpyAsync(&st, status_, sizeof(int), cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
      return cuda_err(err);
    if (st) {
      err = "adjoint run: ";
      if (st & GRAINS_GPU_CONTACT_ERROR) err += "ContactError (overlap exceeded the crust sum); ";
      if (st & GRAINS_GPU_MOTION_ERROR) err += "MotionError (displacement larger than the crust); ";
      if (st & GRAINS_GPU_OUT_OF_GRID) err += "SimulationError (particle outside the grid); ";
      if (st & GRAINS_GPU_HISTORY_FULL) err += "more contacts than contact slots per particle; ";
      if (st & GRAINS_GPU_CUDA_ERROR) err += "internal index error; ";
    }
    return st;
  }
  AdjArgs<R> args() const {
    AdjArgs<R> a{};
    a.n = n_;
    a.cap = cap_;
    a.n_cells = n_cells_;
    a.n_laws = n_laws_;
    a.dt = dt_;
    a.sys = view_.sys;
    a.shapes = view_.shapes;
    a.obs = view_.obs;
    a.cell_obs_start = view_.cell_obs_start;
    a.cell_obs_idx = view_.cell_obs_idx;
    a.laws = (const LawParams<R>*)view_.laws;
    a.md = md_;
    a.meta = meta_;
    a.inertia = inertia_;
    a.cell_count = cell_count_;
    a.cell_start = cell_start_;
    a.block_sums = block_sums_;
    a.perm = perm_;
    a.key = key_;
    a.rank = rank_;
    a.status = status_;
    a.sig = sig_;
    return a;
  }
  AdjState<R> state(int t) const {
    const size_t o = (size_t)t * n_;
    return AdjState<R>{tX_ + o, tV_ + o, tW_ + o};
  }
  AdjRows<R> rows(int t) const {
    const size_t cn = (size_t)cap_ * n_;
    return AdjRows<R>{tcnt_ + (size_t)t * n_, tother_ + (size_t)t * cn, tlink_ + (size_t)t * cn,
                      tmem_ + (size_t)t * 9 * cn};
  }
  // evaluation k from state slot t and rows slot t (previous memory) into
  // rows slot t + 1 and state slot t + 1
  int eval(int k, int t, bool link) {
    AdjArgs<R> a = args();
    if (link) a.sig = sig_ + 2;  // the recomputation hashes into scratch, the run's signature stays
    const int g = grid(n_);
    if (cudaMemsetAsync(cell_count_, 0, (size_t)n_cells_ * sizeof(int), stream_) != cudaSuccess)
      return GRAINS_GPU_CUDA_ERROR;
    adj_bin_kernel<R><<<g, 256, 0, stream_>>>(a, state(t).X);
    const int nb = (n_cells_ + kAdjScanThreads - 1) / kAdjScanThreads;
    adj_scan_blocks<<<nb, kAdjScanThreads, 0, stream_>>>(cell_count_, cell_start_, block_sums_, n_cells_);
    adj_scan_sums<<<1, kAdjScanThreads, 0, stream_>>>(block_sums_, nb, cell_start_, n_cells_);
    adj_scan_add<<<grid(n_cells_), 256, 0, stream_>>>(cell_start_, block_sums_, n_cells_);
    adj_scatter_kernel<R><<<g, 256, 0, stream_>>>(a);
    const R h1 = R(0.5 * dt_);
    const R h2 = (k == 0 || k == K_) ? R(0) : R(0.5 * dt_);
    const int drift = k < K_ ? 1 : 0;
    adj_eval_kernel<R><<<grid(n_, 128), 128, 0, stream_>>>(a, state(t), rows(t), rows(t + 1), state(t + 1), h1, h2,
                                                           drift, k == 0 ? 1 : 0, k);
    if (link) adj_link_kernel<R><<<g, 256, 0, stream_>>>(a, rows(t + 1));
    return cudaGetLastError() == cudaSuccess ? 0 : GRAINS_GPU_CUDA_ERROR;
  }
  int alloc_checkpoints(std::string& err) {
    if (n_seg_ <= ck_count_) return 0;
    for (void* p : ck_pool_) cudaFree(p);
    ck_pool_.clear();
    const size_t N = (size_t)n_, cn = (size_t)cap_ * n_, nck = (size_t)n_seg_;
    void* p[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const size_t b[6] = {nck * N * sizeof(double4), nck * N * sizeof(R4), nck * N * sizeof(R4), nck * N * sizeof(int),
                         nck * cn * sizeof(int), nck * 9 * cn * sizeof(R)};
    for (int k = 0; k < 6; ++k) {
      if (cudaMalloc(&p[k], b[k]) != cudaSuccess) {
        err = "adjoint: not enough device memory for the checkpoints";
        return GRAINS_GPU_CUDA_ERROR;
      }
      ck_pool_.push_back(p[k]);
    }
    cX_ = (double4*)p[0];
    cV_ = (R4*)p[1];
    cW_ = (R4*)p[2];
    ccnt_ = (int*)p[3];
    cother_ = (int*)p[4];
    cmem_ = (R*)p[5];
    ck_count_ = n_seg_;
    return 0;
  }
  int copy(void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream_) == cudaSuccess ? 0
                                                                                               : GRAINS_GPU_CUDA_ERROR;
  }
  // checkpoint j = state slot 0 + rows slot 0 (the memory of the evaluation before)
  int save_checkpoint(int j) {
    const size_t N = (size_t)n_, cn = (size_t)cap_ * n_;
    int rc = copy(cX_ + j * N, tX_, N * sizeof(double4));
    rc |= copy(cV_ + j * N, tV_, N * sizeof(R4));
    rc |= copy(cW_ + j * N, tW_, N * sizeof(R4));
    rc |= copy(ccnt_ + j * N, tcnt_, N * sizeof(int));
    rc |= copy(cother_ + j * cn, tother_, cn * sizeof(int));
    rc |= copy(cmem_ + j * 9 * cn, tmem_, 9 * cn * sizeof(R));
    return rc;
  }
  int restore_checkpoint(int j) {
    const size_t N = (size_t)n_, cn = (size_t)cap_ * n_;
    int rc = copy(tX_, cX_ + j * N, N * sizeof(double4));
    rc |= copy(tV_, cV_ + j * N, N * sizeof(R4));
    rc |= copy(tW_, cW_ + j * N, N * sizeof(R4));
    rc |= copy(tcnt_, ccnt_ + j * N, N * sizeof(int));
    rc |= copy(tother_, cother_ + j * cn, cn * sizeof(int));
    rc |= copy(tmem_, cmem_ + j * 9 * cn, 9 * cn * sizeof(R));
    return rc;
  }
  // slot t -> slot 0 (the start of the next segment)
  int shift_slot(int t) {
    const size_t N = (size_t)n_, cn = (size_t)cap_ * n_;
    int rc = copy(tX_, tX_ + t * N, N * sizeof(double4));
    rc |= copy(tV_, tV_ + t * N, N * sizeof(R4));
    rc |= copy(tW_, tW_ + t * N, N * sizeof(R4));
    rc |= copy(tcnt_, tcnt_ + t * N, N * sizeof(int));
    rc |= copy(tother_, tother_ + t * cn, cn * sizeof(int));
    rc |= copy(tmem_, tmem_ + t * 9 * cn, 9 * cn * sizeof(R));
    return rc;
  }

  int n_ = 0, cap_ = 0, S_ = 1, n_cells_ = 0, n_laws_ = 0;
  int K_ = 0, n_seg_ = 0, ck_count_ = 0, last_len_ = 0;
  double dt_ = 0.;
  bool ok_ = true, have_forward_ = false;
  size_t bytes_ = 0;
  cudaStream_t stream_ = nullptr;
  ContextView view_{};
  std::vector<void*> pool_, ck_pool_;
  double4* md_ = nullptr;
  int4* meta_ = nullptr;
  R* inertia_ = nullptr;
  int *cell_count_ = nullptr, *cell_start_ = nullptr, *block_sums_ = nullptr, *perm_ = nullptr, *status_ = nullptr;
  unsigned long long* sig_ = nullptr;
  unsigned long long sig_host_[2] = {0ull, 0ull};
  unsigned *key_ = nullptr, *rank_ = nullptr;
  double4* tX_ = nullptr;
  R4 *tV_ = nullptr, *tW_ = nullptr;
  int *tcnt_ = nullptr, *tother_ = nullptr, *tlink_ = nullptr;
  R* tmem_ = nullptr;
  double4* cX_ = nullptr;
  R4 *cV_ = nullptr, *cW_ = nullptr;
  int *ccnt_ = nullptr, *cother_ = nullptr;
  R* cmem_ = nullptr;
  R* lam_[2] = {nullptr, nullptr};
  R* radj_ = nullptr;
  R4 *aX_ = nullptr, *aV_ = nullptr, *aW_ = nullptr, *aF_ = nullptr, *aT_ = nullptr;
  double *gtheta_ = nullptr, *theta_ = nullptr, *gin_ = nullptr, *gout_ = nullptr;
};

template <typename R, int LANES>
AdjointEngine* make_adjoint_engine(const ContextView& v, int checkpoint_every, std::string& err) {
  auto* e = new AdjEngineT<R, LANES>(v, checkpoint_every);
  if (!e->ok()) {
    delete e;
    err = "adjoint: not enough device memory for the tape";
    return nullptr;
  }
  return e;
}

}  // namespace gg
