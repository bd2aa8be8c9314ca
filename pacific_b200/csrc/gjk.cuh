// gjk.cuh -- closest points of two convex bodies with crust by the Johnson
// GJK distance algorithm (van den Bergen, "A fast and robust GJK
// implementation for collision detection of convex objects", J. Graphics
// Tools 4(2), 1999: Johnson's sub-algorithm with cached sub-determinants and
// the backup procedure).  Behaviour follows the reference's closest_points
// (Geometry/src/Convex.cpp:536-627): same start point, same termination tests
// (relative / absolute optimality gap, degenerate support point, full simplex,
// distance <= EPSILON2, 1000 iterations) so that iteration counts and witness
// points match.
//
// Support functions: Sphere.cpp:99-109, Box.cpp:307-316, Cylinder.cpp:112-133
// (axis = local Y), Polyhedron.cpp:265-293.  The polyhedron support climbs the
// vertex adjacency like the reference: from the current vertex to the first
// neighbour (in adjacency order) that raises v . p by at least 1e-16, until no
// neighbour does.  The reference keeps the current vertex per body between GJK
// runs; here every GJK run starts its climb at vertex 0 and carries the vertex
// from one support call to the next within the run.  On flat faces the vertex
// reached depends on where the climb starts; over every polyhedron fixture and
// a 1,500-step dense run of cubes, cylinders and octahedra the two rules gave
// identical results, while the order-independent arg-max (kept for bodies
// without adjacency) moved contact points by up to 3e-4 of the weight.
//
// Options of <CollisionDetection> (Base/src/Grains.cpp:654-723), passed in a
// GjkStart: the tolerance of the optimality gap, the Nesterov-accelerated
// search direction (Acceleration="ON": momentum k / (k + 2) on the direction,
// plain every 8th iteration, and on convergence either stop, when the
// accelerated direction has met the plain one, or go on without momentum --
// the rule of Montaut et al., "Collision detection accelerated: an
// optimization perspective", RSS 2022, as Convex.cpp:566-597 applies it), and
// the warm start of History="ON" (Convex.cpp:636-716): the run starts from a
// given direction v0 (its first support point in -v0), or from A(0) - B(0)
// when there is none, with the distance estimate set to 1.
//
// Precision: the iteration runs in T; the step kernels of both precisions use
// T = double (an FP32 run is too inaccurate for contact features and was
// slower on B200, see convex_closest_point in kernels.cuh).  With T = float
// the two bodies are expressed relative to body A's origin so that FP32 keeps
// the body-size scale; GjkResult::lower is a lower bound of the distance.
#pragma once

#include "common.cuh"
#include "device_state.h"
#include "sphere_contact.cuh"

namespace gg {

struct BodyRef {
  int type;
  int nverts;
  const double* verts;
  double radius;       // sphere radius / circumscribed radius
  double cyl_r, cyl_hh;
  D3 ext;              // box half edges
  double crust;
  M3 basis;            // rotation part
  D3 origin;
  double scaling[3];   // crust shrink factors (RigidBodyWithCrust.cpp:60-72)
  double lext[3];      // local bounding-box half extents (Convex::bbox with identity)
  // polyhedron vertex adjacency (Polyhedron::m_cobound): the neighbours of
  // vertex i are adj[adj_start[i] .. adj_start[i + 1]); nullptr: arg-max support
  const int* adj_start = nullptr;
  const int* adj = nullptr;
};

template <typename T>
struct LocalBody {
  int type;
  int nverts;
  const double* verts;
  T radius, cyl_r, cyl_hh;
  V3<T> ext;
  T b[9];   // shrunk basis
  V3<T> o;  // origin in the working frame
  const int* adj_start = nullptr;  // polyhedron adjacency (see BodyRef)
  const int* adj = nullptr;
  mutable int cur = 0;  // the hill climb's current vertex, carried between support calls
};

template <typename T>
GG_HD V3<T> support_local(const LocalBody<T>& B, V3<T> v) {
  switch (B.type) {
    case 0: {  // sphere
      T s = norm(v);
      if (s > T(kEpsilon)) {
        T r = B.radius / s;
        return v3<T>(v.x * r, v.y * r, v.z * r);
      }
      return v3<T>(T(0), T(0), T(0));
    }
    case 1: {  // box
      // |v| < EPSILON tested as |v|^2 < EPSILON^2 here and below: the same
      // branch except within a rounding of the threshold, without the square
      // root (two per GJK iteration)
      if (norm2(v) < T(kEpsilon) * T(kEpsilon)) return v3<T>(T(0), T(0), T(0));
      return v3<T>(v.x < T(0) ? -B.ext.x : B.ext.x, v.y < T(0) ? -B.ext.y : B.ext.y,
                   v.z < T(0) ? -B.ext.z : B.ext.z);
    }
    case 2: {  // cylinder, axis local Y
      if (norm2(v) > T(kEpsilon) * T(kEpsilon)) {
        T s = std::sqrt(v.x * v.x + v.z * v.z);
        if (s > T(kEpsilon)) {
          T d = B.cyl_r / s;
          if (std::fabs(v.y) < T(kEpsilon)) return v3<T>(v.x * d, T(0), v.z * d);
          return v3<T>(v.x * d, v.y < T(0) ? -B.cyl_hh : B.cyl_hh, v.z * d);
        }
        return v3<T>(T(0), v.y < T(0) ? -B.cyl_hh : B.cyl_hh, T(0));
      }
      return v3<T>(T(0), T(0), T(0));
    }
    default: {  // polyhedron
      if (!(norm2(v) > T(kEpsilon) * T(kEpsilon))) return v3<T>(T(0), T(0), T(0));
      if (B.adj_start) {
        // hill climb: move to the first neighbour (other than the vertex just
        // left) whose v . p is not below the current one by the 1e-16 margin;
        // every move raises v . p, so at most nverts moves (the bound also
        // ends the climb when v holds a NaN)
        int cur = B.cur, last = -1;
        T h = dot(v3<T>(T(B.verts[3 * cur]), T(B.verts[3 * cur + 1]), T(B.verts[3 * cur + 2])), v);
        for (int moves = 0; moves < B.nverts; ++moves) {
          int next = -1;
          T dn = T(0);
          for (int k = B.adj_start[cur]; k < B.adj_start[cur + 1]; ++k) {
            const int c = B.adj[k];
            if (c == last) continue;
            const T d = dot(v3<T>(T(B.verts[3 * c]), T(B.verts[3 * c + 1]), T(B.verts[3 * c + 2])), v);
            if (!(d - h < T(1.e-16))) {
              next = c;
              dn = d;
              break;
            }
          }
          if (next < 0) break;
          last = cur;
          cur = next;
          h = dn;
        }
        B.cur = cur;
        return v3<T>(T(B.verts[3 * cur]), T(B.verts[3 * cur + 1]), T(B.verts[3 * cur + 2]));
      }
      int best = 0;
      V3<T> p0 = v3<T>(T(B.verts[0]), T(B.verts[1]), T(B.verts[2]));
      T h = dot(p0, v);
      for (int i = 1; i < B.nverts; ++i) {
        V3<T> p = v3<T>(T(B.verts[3 * i]), T(B.verts[3 * i + 1]), T(B.verts[3 * i + 2]));
        T d = dot(p, v);
        if (d > h) {
          h = d;
          best = i;
        }
      }
      return v3<T>(T(B.verts[3 * best]), T(B.verts[3 * best + 1]), T(B.verts[3 * best + 2]));
    }
  }
}

template <typename T>
GG_HD V3<T> lb_apply(const LocalBody<T>& B, V3<T> p) {
  return v3<T>(B.b[0] * p.x + B.b[1] * p.y + B.b[2] * p.z + B.o.x,
               B.b[3] * p.x + B.b[4] * p.y + B.b[5] * p.z + B.o.y,
               B.b[6] * p.x + B.b[7] * p.y + B.b[8] * p.z + B.o.z);
}
template <typename T>
GG_HD V3<T> lb_vecmat(V3<T> v, const LocalBody<T>& B) {  // v * basis
  return v3<T>(B.b[0] * v.x + B.b[3] * v.y + B.b[6] * v.z, B.b[1] * v.x + B.b[4] * v.y + B.b[7] * v.z,
               B.b[2] * v.x + B.b[5] * v.y + B.b[8] * v.z);
}

// Builds the working-frame body (crust-shrunk basis, origin relative to 'shift')
template <typename T>
GG_HD LocalBody<T> local_body(const BodyRef& r, D3 shift, const double scale[3]) {
  LocalBody<T> B;
  B.type = r.type;
  B.nverts = r.nverts;
  B.verts = r.verts;
  B.radius = T(r.radius);
  B.cyl_r = T(r.cyl_r);
  B.cyl_hh = T(r.cyl_hh);
  B.ext = v3<T>(T(r.ext.x), T(r.ext.y), T(r.ext.z));
  M3 s = mscale_cols(r.basis, scale[0], scale[1], scale[2]);
  for (int i = 0; i < 9; ++i) B.b[i] = T(s.m[i]);
  D3 o = xsub3(r.origin, shift);
  B.o = v3<T>(T(o.x), T(o.y), T(o.z));
  B.adj_start = r.adj_start;
  B.adj = r.adj;
  B.cur = 0;
  return B;
}

// How a GJK run starts and searches (the options of <CollisionDetection>)
template <typename T>
struct GjkStart {
  bool accel = false;    // Nesterov-accelerated search direction
  bool history = false;  // warm-started run: distance estimate 1, first direction v0 (when non-zero)
  V3<T> v0 = {T(0), T(0), T(0)};
};

// The first iterate of a run: v and the support point w that goes with it,
// and the distance estimate (Convex.cpp:557-561 plain, :659-668 warm-started).
template <typename T>
GG_HD T gjk_first(const LocalBody<T>& A, const LocalBody<T>& B, const GjkStart<T>& st, V3<T>& v, V3<T>& w) {
  const V3<T> zero = v3<T>(T(0), T(0), T(0));
  if (st.history && !(st.v0.x == T(0) && st.v0.y == T(0) && st.v0.z == T(0))) {
    v = st.v0;
    w = lb_apply(A, support_local(A, lb_vecmat(-v, A))) - lb_apply(B, support_local(B, lb_vecmat(v, B)));
  } else {
    v = lb_apply(A, support_local(A, zero)) - lb_apply(B, support_local(B, zero));
    w = v;
  }
  return st.history ? T(1) : norm(v);
}

// The search direction of iteration k: with acceleration (except every 8th
// iteration) d = m d + m (1 - m) v + (1 - m)^2 w with m = k / (k + 2), else v.
template <typename T>
GG_HD V3<T> gjk_direction(bool accel, int k, V3<T> d, V3<T> v, V3<T> w) {
  if (accel && k % 8 != 0) {
    const T m = T(k) / (T(k) + T(2));
    const T om = T(1) - m;
    return sc(d, m) + sc(v, m * om) + sc(w, om * om);
  }
  return v;
}

// The arrays of a Johnson GJK run, as a view of kGjkWords numbers `stride`
// apart: the sub-determinants of every subset s of the 4-point simplex for
// each of its points i (32 values, packed by subset: the entries of s start at
// the number of point slots of the subsets below it), the dot products of the
// simplex points (16), the points of A - B, and the support points of A and B
// in their local frames (3 x 4 x 3).  A run on its own keeps them in a local
// array (stride 1); the GJK kernel keeps those of its 64 threads interleaved
// in shared memory (stride 64), so that a warp's accesses fall in distinct
// banks.
constexpr int kGjkWords = 32 + 16 + 36;
template <typename T>
struct GjkState {
  T* base;
  int stride;
  GG_HD static int at(unsigned s, unsigned i) {
    // sum of the sizes of the subsets 0 .. s-1, bytes of two constants
    const unsigned long long lo = 0x0907050402010000ull, hi = 0x1C191614110F0D0Cull;
    const unsigned start = unsigned((s < 8 ? lo >> (8 * s) : hi >> (8 * (s - 8))) & 0xffu);
#if defined(__CUDA_ARCH__)
    return int(start + __popc(s & ((1u << i) - 1u)));
#else
    return int(start + __builtin_popcount(s & ((1u << i) - 1u)));
#endif
  }
  GG_HD T& det(unsigned s, unsigned i) const { return base[at(s, i) * stride]; }
  GG_HD T& dp(unsigned i, unsigned j) const { return base[(32 + 4 * i + j) * stride]; }
  GG_HD V3<T> vec(int k) const {  // k: 0-3 y, 4-7 p, 8-11 q
    const T* b = base + (48 + 3 * k) * stride;
    return v3<T>(b[0], b[stride], b[2 * stride]);
  }
  GG_HD void set_vec(int k, V3<T> v) const {
    T* b = base + (48 + 3 * k) * stride;
    b[0] = v.x;
    b[stride] = v.y;
    b[2 * stride] = v.z;
  }
  GG_HD V3<T> y(unsigned i) const { return vec(int(i)); }
  GG_HD V3<T> p(unsigned i) const { return vec(4 + int(i)); }
  GG_HD V3<T> q(unsigned i) const { return vec(8 + int(i)); }
};

template <typename T>
GG_HD void gjk_det(unsigned bits, unsigned last, unsigned last_bit, unsigned all_bits, const GjkState<T>& g) {
  const V3<T> yl = g.y(last);
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (bits & bit) g.dp(i, last) = g.dp(last, i) = dot(g.y(i), yl);
  g.dp(last, last) = dot(yl, yl);
  g.det(last_bit, last) = T(1);
  for (unsigned j = 0, sj = 1; j < 4; ++j, sj <<= 1) {
    if (!(bits & sj)) continue;
    unsigned s2 = sj | last_bit;
    g.det(s2, j) = g.dp(last, last) - g.dp(last, j);
    g.det(s2, last) = g.dp(j, j) - g.dp(j, last);
    for (unsigned k = 0, sk = 1; k < j; ++k, sk <<= 1) {
      if (!(bits & sk)) continue;
      unsigned s3 = sk | s2;
      g.det(s3, k) = g.det(s2, j) * (g.dp(j, j) - g.dp(j, k)) + g.det(s2, last) * (g.dp(last, j) - g.dp(last, k));
      g.det(s3, j) = g.det(sk | last_bit, k) * (g.dp(k, k) - g.dp(k, j)) +
                     g.det(sk | last_bit, last) * (g.dp(last, k) - g.dp(last, j));
      g.det(s3, last) = g.det(sk | sj, k) * (g.dp(k, k) - g.dp(k, last)) +
                        g.det(sk | sj, j) * (g.dp(j, k) - g.dp(j, last));
    }
  }
  if (all_bits == 15) {
    g.det(15, 0) = g.det(14, 1) * (g.dp(1, 1) - g.dp(1, 0)) + g.det(14, 2) * (g.dp(2, 1) - g.dp(2, 0)) +
                   g.det(14, 3) * (g.dp(3, 1) - g.dp(3, 0));
    g.det(15, 1) = g.det(13, 0) * (g.dp(0, 0) - g.dp(0, 1)) + g.det(13, 2) * (g.dp(2, 0) - g.dp(2, 1)) +
                   g.det(13, 3) * (g.dp(3, 0) - g.dp(3, 1));
    g.det(15, 2) = g.det(11, 0) * (g.dp(0, 0) - g.dp(0, 2)) + g.det(11, 1) * (g.dp(1, 0) - g.dp(1, 2)) +
                   g.det(11, 3) * (g.dp(3, 0) - g.dp(3, 2));
    g.det(15, 3) = g.det(7, 0) * (g.dp(0, 0) - g.dp(0, 3)) + g.det(7, 1) * (g.dp(1, 0) - g.dp(1, 3)) +
                   g.det(7, 2) * (g.dp(2, 0) - g.dp(2, 3));
  }
}

template <typename T>
GG_HD bool gjk_valid(unsigned s, unsigned all_bits, const GjkState<T>& g) {
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1) {
    if (!(all_bits & bit)) continue;
    if (s & bit) {
      if (g.det(s, i) <= T(kEpsilon3)) return false;
    } else if (g.det(s | bit, i) > T(0)) {
      return false;
    }
  }
  return true;
}

template <typename T>
GG_HD V3<T> gjk_vector(unsigned bits, const GjkState<T>& g) {
  T sum = T(0);
  V3<T> v = v3<T>(T(0), T(0), T(0));
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (bits & bit) {
      sum += g.det(bits, i);
      v = v + sc(g.y(i), g.det(bits, i));
    }
  return sc(v, T(1) / sum);
}

template <typename T>
GG_HD bool gjk_proper(unsigned s, const GjkState<T>& g) {
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if ((s & bit) && g.det(s, i) <= T(kEpsilon3)) return false;
  return true;
}

template <typename T>
GG_HD bool gjk_closest(unsigned& bits, unsigned last, unsigned last_bit, unsigned all_bits, const GjkState<T>& g,
                       V3<T>& v) {
  gjk_det(bits, last, last_bit, all_bits, g);
  // the non-empty subsets of bits in decreasing order (s = (s - 1) & bits
  // steps from one subset to the next smaller one)
  for (unsigned s = bits; s; s = (s - 1) & bits) {
    if (gjk_valid(s | last_bit, all_bits, g)) {
      bits = s | last_bit;
      v = gjk_vector(bits, g);
      return true;
    }
  }
  if (gjk_valid(last_bit, all_bits, g)) {
    bits = last_bit;
    v = g.y(last);
    return true;
  }
  T best = T(INFINITY);
  for (unsigned s = all_bits; s; s = (s - 1) & all_bits) {  // backup procedure
    if (gjk_proper(s, g)) {
      V3<T> u = gjk_vector(s, g);
      T d2 = norm2(u);
      if (d2 < best) {
        best = d2;
        bits = s;
        v = u;
      }
    }
  }
  return false;
}

template <typename T>
struct GjkResult {
  T dist;
  V3<T> pa, pb;  // witness points in the working frame
  int iters;
  T lower;   // largest support-plane separation dot(v, w) / |v| met: a lower bound of the distance
  int exit;  // 0 optimality gap, 1 degenerate support point, 2 Johnson/backup failed, 3 other (full simplex,
             // distance <= EPSILON2, iteration cap)
  V3<T> v;   // the last iterate (the direction a warm-started run keeps for the pair)
};

// The Johnson GJK run as a resumable state: gjk_begin sets up the first
// iterate, gjk_iterate performs one pass of the loop of closest_points
// (Convex.cpp:563-618) and says whether the run has ended, gjk_end forms the
// witness points.  gjk_distance strings them together; the lane-persistent GJK
// kernel interleaves the passes of different pairs on one thread.
template <typename T>
struct GjkRun {
  unsigned bits, last, last_bit, all_bits;
  GjkState<T> g;  // the run's arrays (the caller's storage)
  V3<T> v, w, d;
  T dist, lower, rel_error, abs_error;
  int num, exit_reason;
  bool accel;
};

template <typename T>
GG_HD void gjk_begin(GjkRun<T>& r, const LocalBody<T>& A, const LocalBody<T>& B, T rel_error,
                     const GjkStart<T>& st) {
  r.bits = r.last = r.last_bit = r.all_bits = 0;
  for (int i = 0; i < kGjkWords; ++i) r.g.base[i * r.g.stride] = T(0);
  r.rel_error = rel_error;
  r.abs_error = T(1.e-4) * rel_error;
  r.dist = gjk_first(A, B, st, r.v, r.w);
  r.d = r.v;
  r.accel = st.accel;
  r.num = 0;
  r.exit_reason = 3;
  r.lower = -r.dist;
}

// one pass of the loop; true when the run has ended
template <typename T>
GG_HD bool gjk_iterate(GjkRun<T>& r, const LocalBody<T>& A, const LocalBody<T>& B) {
  if (!(r.bits < 15 && r.dist > T(kEpsilon2) && r.num < 1000)) return true;
  ++r.num;
  r.last = 0;
  r.last_bit = 1;
  while (r.bits & r.last_bit) {
    ++r.last;
    r.last_bit <<= 1;
  }
  const unsigned last = r.last;
  r.d = gjk_direction(r.accel, r.num, r.d, r.v, r.w);
  V3<T> pl = support_local(A, lb_vecmat(-r.d, A));
  V3<T> ql = support_local(B, lb_vecmat(r.d, B));
  r.w = lb_apply(A, pl) - lb_apply(B, ql);
  const T sep = dot(r.v, r.w) / r.dist;
  if (sep > r.lower) r.lower = sep;
  T mu = r.dist - sep;
  if (mu < r.dist * r.rel_error || mu < r.abs_error) {
    if (!r.accel || norm(r.d - r.v) < T(kEpsilon)) {
      r.g.set_vec(4 + int(last), pl);
      r.g.set_vec(8 + int(last), ql);
      r.exit_reason = 0;
      return true;
    }
    // converged on the accelerated direction only: go on without momentum
    r.accel = false;
    pl = support_local(A, lb_vecmat(-r.v, A));
    ql = support_local(B, lb_vecmat(r.v, B));
    r.w = lb_apply(A, pl) - lb_apply(B, ql);
  }
  r.g.set_vec(4 + int(last), pl);
  r.g.set_vec(8 + int(last), ql);
  bool degen = false;
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (r.all_bits & bit) {
      const V3<T> yi = r.g.y(i);
      if (yi.x == r.w.x && yi.y == r.w.y && yi.z == r.w.z) degen = true;
    }
  if (degen) {
    r.exit_reason = 1;
    return true;
  }
  r.g.set_vec(int(last), r.w);
  r.all_bits = r.bits | r.last_bit;
  if (!gjk_closest(r.bits, last, r.last_bit, r.all_bits, r.g, r.v)) {
    r.exit_reason = 2;
    return true;
  }
  r.dist = norm(r.v);
  return false;
}

template <typename T>
GG_HD GjkResult<T> gjk_end(const GjkRun<T>& r, const LocalBody<T>& A, const LocalBody<T>& B) {
  GjkResult<T> out;
  T sum = T(0);
  const V3<T> zero = v3<T>(T(0), T(0), T(0));
  V3<T> pa = zero, pb = zero;
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (r.bits & bit) {
      const T di = r.g.det(r.bits, i);
      sum += di;
      pa = pa + sc(r.g.p(i), di);
      pb = pb + sc(r.g.q(i), di);
    }
  T s = T(1) / sum;
  out.pa = lb_apply(A, sc(pa, s));
  out.pb = lb_apply(B, sc(pb, s));
  out.dist = r.dist;
  out.iters = r.num;
  out.exit = r.exit_reason;
  out.lower = r.lower;
  out.v = r.v;
  return out;
}

template <typename T>
GG_HD GjkResult<T> gjk_distance(const LocalBody<T>& A, const LocalBody<T>& B, T rel_error,
                                const GjkStart<T>& st = GjkStart<T>()) {
  T words[kGjkWords];
  GjkRun<T> r;
  r.g.base = words;
  r.g.stride = 1;
  gjk_begin(r, A, B, rel_error, st);
  while (!gjk_iterate(r, A, B)) {
  }
  return gjk_end(r, A, B);
}

// ---- the signed-volume GJK ------------------------------------------------------
// Montanari, Petrinic and Barbieri, "Improving the GJK algorithm for faster and
// more reliable distance queries between convex objects", ACM Transactions on
// Graphics 36(3), 2017.  Its distance sub-algorithm finds the point of a
// simplex W = {y_k} closest to the origin from signed volumes: the barycentric
// coordinate of y_k in the origin's projection onto aff(W) is the signed volume
// of W with y_k replaced by that projection, over the signed volume of W.  When
// every such volume has the sign of the whole, the projection lies inside W and
// is the answer.  Otherwise each face of W opposite a vertex whose volume has
// the wrong sign is searched in turn (one dimension lower), and the closest of
// their answers is kept.
//
// Formulation used here (vector products over the full 3-vectors, no
// projection onto a coordinate plane), with edge vectors taken between
// vertices wherever possible: near convergence the simplex is far smaller than
// its distance from the origin, and products of the vertices themselves would
// cancel to rounding noise.
//   segment (a, b):      t = b - a; the projection's signed length past a is
//                        u = -a.t (in units of 1 / |t|); weights (t.t - u, u) / t.t
//   triangle (a, b, c):  n = (b - a) x (c - a), p = the origin's projection onto
//                        the plane; the signed areas measured along n are
//                        n.((b - p) x (c - p)) and cyclically (total n.n)
//   tetrahedron:         the volume with y_k replaced by the origin, e.g.
//                        det[y1, y2 - y1, y3 - y1] for y0, with alternating
//                        signs; the whole: det[y1 - y0, y2 - y0, y3 - y0]
// A zero volume counts as a wrong sign, so a projection on the boundary of W is
// answered by the smaller simplex.  The simplex is kept packed: vertices
// 0 .. n-1, the newest last.

// closest point of a sub-simplex: the vertices kept (bit k = vertex k) and
// their weights, and the squared distance of the point from the origin
struct SvPick {
  unsigned keep;
  double lam[4];
  double d2;
};

GG_HD double sv_triple(V3<double> a, V3<double> b, V3<double> c) { return dot(a, cross(b, c)); }

GG_HD void sv_finish(const V3<double>* y, SvPick& r) {
  V3<double> pt = v3<double>(0., 0., 0.);
  for (int k = 0; k < 4; ++k)
    if (r.keep & (1u << k)) pt = pt + sc(y[k], r.lam[k]);
  r.d2 = dot(pt, pt);
}

GG_HD SvPick sv_pick_vertex(const V3<double>* y, int a) {
  SvPick r{1u << a, {0., 0., 0., 0.}, 0.};
  r.lam[a] = 1.;
  r.d2 = dot(y[a], y[a]);
  return r;
}

GG_HD SvPick sv_pick_segment(const V3<double>* y, int a, int b) {
  const V3<double> t = y[b] - y[a];
  const double tt = dot(t, t);
  const double u = -dot(y[a], t);
  if (!(u > 0.)) return sv_pick_vertex(y, a);        // the origin projects before a
  if (!(u < tt)) return sv_pick_vertex(y, b);        // ... past b (or a, b coincide)
  SvPick r{(1u << a) | (1u << b), {0., 0., 0., 0.}, 0.};
  r.lam[b] = u / tt;
  r.lam[a] = (tt - u) / tt;
  sv_finish(y, r);
  return r;
}

GG_HD SvPick sv_pick_triangle(const V3<double>* y, int a, int b, int c) {
  const V3<double> n = cross(y[b] - y[a], y[c] - y[a]);
  const double nn = dot(n, n);
  const int vx[3] = {a, b, c};
  double area[3] = {0., 0., 0.};
  if (nn > 0.) {
    const V3<double> p = sc(n, dot(n, y[a]) / nn);
    area[0] = dot(n, cross(y[b] - p, y[c] - p));
    area[1] = dot(n, cross(y[c] - p, y[a] - p));
    area[2] = dot(n, cross(y[a] - p, y[b] - p));
  }
  if (area[0] > 0. && area[1] > 0. && area[2] > 0.) {
    const double total = area[0] + area[1] + area[2];
    SvPick r{(1u << a) | (1u << b) | (1u << c), {0., 0., 0., 0.}, 0.};
    for (int k = 0; k < 3; ++k) r.lam[vx[k]] = area[k] / total;
    sv_finish(y, r);
    return r;
  }
  SvPick best{0u, {0., 0., 0., 0.}, INFINITY};
  for (int k = 0; k < 3; ++k) {
    if (area[k] > 0.) continue;  // the projection is on y_k's side of the opposite edge
    const SvPick e = sv_pick_segment(y, vx[(k + 1) % 3], vx[(k + 2) % 3]);
    if (e.d2 < best.d2) best = e;
  }
  return best;
}

GG_HD SvPick sv_pick_tetrahedron(const V3<double>* y) {
  const double vol[4] = {sv_triple(y[1], y[2] - y[1], y[3] - y[1]), -sv_triple(y[0], y[2] - y[0], y[3] - y[0]),
                         sv_triple(y[0], y[1] - y[0], y[3] - y[0]), -sv_triple(y[0], y[1] - y[0], y[2] - y[0])};
  const double total = sv_triple(y[1] - y[0], y[2] - y[0], y[3] - y[0]);
  bool same[4];
  for (int k = 0; k < 4; ++k) same[k] = vol[k] != 0. && ((vol[k] > 0.) == (total > 0.));
  if (total != 0. && same[0] && same[1] && same[2] && same[3]) {
    const double sum = (vol[0] + vol[1]) + (vol[2] + vol[3]);
    SvPick r{15u, {vol[0] / sum, vol[1] / sum, vol[2] / sum, vol[3] / sum}, 0.};
    return r;  // the origin is inside: distance zero
  }
  SvPick best{0u, {0., 0., 0., 0.}, INFINITY};
  for (int k = 0; k < 4; ++k) {
    if (same[k] && total != 0.) continue;
    const SvPick f = sv_pick_triangle(y, (k + 1) & 3, (k + 2) & 3, (k + 3) & 3);
    if (f.d2 < best.d2) best = f;
  }
  return best;
}

// GJK iteration with the signed-volume sub-algorithm.  The outer loop follows
// the reference's closest_points_GJK_SV (GJK_SV.cpp:428-631): start at
// A(0) - B(0) or from a warm-start direction, stop on the optimality gap
// (relative rel_error or absolute 1e-4 rel_error), on a support point already
// in the simplex, on a full simplex, at distance <= EPSILON2 or after 1000
// iterations; the accelerated direction as in gjk_distance.
GG_HD GjkResult<double> gjk_sv_distance(const LocalBody<double>& A, const LocalBody<double>& B, double rel_error,
                                        const GjkStart<double>& st = GjkStart<double>()) {
  const V3<double> zero = v3<double>(0., 0., 0.);
  V3<double> y[4], p[4], q[4];
  double lam[4] = {0., 0., 0., 0.};
  for (int i = 0; i < 4; ++i) y[i] = p[i] = q[i] = zero;
  int n = 0;  // vertices in the simplex
  const double abs_error = 1.e-4 * rel_error;
  V3<double> v, w;
  double dist = gjk_first(A, B, st, v, w);
  V3<double> d = v;
  bool accel = st.accel;
  int iters = 0, exit_reason = 3;
  double lower = -dist;
  while (n < 4 && dist > kEpsilon2 && iters < 1000) {
    ++iters;
    d = gjk_direction(accel, iters, d, v, w);
    V3<double> pa = support_local(A, lb_vecmat(-d, A));
    V3<double> qb = support_local(B, lb_vecmat(d, B));
    w = lb_apply(A, pa) - lb_apply(B, qb);
    const double sep = dot(v, w) / dist;
    if (sep > lower) lower = sep;
    const double gap = dist - sep;
    if (gap < dist * rel_error || gap < abs_error) {
      if (!accel || norm(d - v) < kEpsilon) {
        exit_reason = 0;
        break;
      }
      accel = false;
      pa = support_local(A, lb_vecmat(-v, A));
      qb = support_local(B, lb_vecmat(v, B));
      w = lb_apply(A, pa) - lb_apply(B, qb);
    }
    bool repeated = false;
    for (int k = 0; k < n; ++k) repeated = repeated || (y[k].x == w.x && y[k].y == w.y && y[k].z == w.z);
    if (repeated) {
      exit_reason = 1;
      break;
    }
    y[n] = w;
    p[n] = pa;
    q[n] = qb;
    ++n;
    SvPick pick;
    if (n == 1) pick = sv_pick_vertex(y, 0);
    else if (n == 2) pick = sv_pick_segment(y, 0, 1);
    else if (n == 3) pick = sv_pick_triangle(y, 0, 1, 2);
    else pick = sv_pick_tetrahedron(y);
    // In exact arithmetic the new support point is part of the answer whenever
    // the optimality gap is still open; when rounding drops it, the next
    // iteration would find the same point again and cycle: stop here, with the
    // answer of the current simplex (like a support point already in it).
    const bool dropped = !(pick.keep & (1u << (n - 1)));
    // pack the kept vertices to the front, in their order
    int m = 0;
    v = zero;
    for (int k = 0; k < n; ++k) {
      if (!(pick.keep & (1u << k))) continue;
      y[m] = y[k];
      p[m] = p[k];
      q[m] = q[k];
      lam[m] = pick.lam[k];
      v = v + sc(y[m], lam[m]);
      ++m;
    }
    n = m;
    dist = norm(v);
    if (dropped) {
      exit_reason = 1;
      break;
    }
  }
  V3<double> wa = zero, wb = zero;
  for (int k = 0; k < n; ++k) {
    wa = wa + sc(p[k], lam[k]);
    wb = wb + sc(q[k], lam[k]);
  }
  GjkResult<double> r;
  r.pa = lb_apply(A, wa);
  r.pb = lb_apply(B, wb);
  r.dist = dist;
  r.iters = iters;
  r.exit = exit_reason;
  r.lower = lower;
  r.v = v;
  return r;
}

// The contact features of a finished distance run (RigidBodyWithCrust.cpp:
// 314-348): status 1 (ContactError) when the crust-shrunk bodies touch, else
// the contact point midway between the witness points, the overlap vector
// along B -> A, and the overlap distance - crust_a - crust_b.
template <typename T>
GG_HD ContactGeom gjk_features(const GjkResult<T>& r, double crust_sum, D3 shift) {
  ContactGeom c = no_contact();
  double distance = double(r.dist);
  if (distance < kEpsilon) {
    c.status = 1;
    return c;
  }
  V3<T> ba = r.pa - r.pb;
  V3<T> pc = dv(r.pa, T(2)) + dv(r.pb, T(2));
  V3<T> ov = round3(dv(ba, r.dist));
  ov = sc(ov, T(crust_sum) - r.dist);
  c.point = xadd3(d3(double(pc.x), double(pc.y), double(pc.z)), shift);
  c.overlap_vector = d3(double(ov.x), double(ov.y), double(ov.z));
  c.overlap = distance - crust_sum;
  c.status = 0;
  return c;
}

// RigidBodyWithCrust::ClosestPoint general case (RigidBodyWithCrust.cpp:278-348).
// status: 0 = features valid, 1 = ContactError, 2 = bounding spheres apart.
// With a GjkStart, st->v0 on return holds the run's last iterate (the
// direction RigidBodyWithCrust::ClosestPoint hands back to the collision
// history, RigidBodyWithCrust.cpp:362-470), or zero when the bounding spheres
// are apart (:510-514).
template <typename T>
GG_HD ContactGeom convex_closest_point_t(const BodyRef& A, const BodyRef& B, double tol, int* iters,
                                        int* exit_out = nullptr, double* lower_out = nullptr,
                                        GjkStart<T>* st = nullptr) {
  ContactGeom c = no_contact();
  D3 g = xsub3(A.origin, B.origin);
  if (!(xnorm(g) < xadd(A.radius, B.radius))) {
    c.status = 2;
    if (st) st->v0 = v3<T>(T(0), T(0), T(0));
    return c;
  }
  const D3 shift = sizeof(T) == 4 ? A.origin : d3(0., 0., 0.);
  LocalBody<T> la = local_body<T>(A, shift, A.scaling);
  LocalBody<T> lb = local_body<T>(B, shift, B.scaling);
  GjkResult<T> r = st ? gjk_distance(la, lb, T(tol), *st) : gjk_distance(la, lb, T(tol));
  if (st) st->v0 = r.v;
  *iters = r.iters;
  if (exit_out) *exit_out = r.exit;
  if (lower_out) *lower_out = double(r.lower);
  return gjk_features(r, xadd(A.crust, B.crust), shift);
}

// RigidBodyWithCrust::ClosestPoint with the signed-volume GJK (the same
// features as convex_closest_point_t)
GG_HD ContactGeom convex_closest_point_sv(const BodyRef& A, const BodyRef& B, double tol, int* iters,
                                         GjkStart<double>* st = nullptr) {
  ContactGeom c = no_contact();
  D3 g = xsub3(A.origin, B.origin);
  if (!(xnorm(g) < xadd(A.radius, B.radius))) {
    c.status = 2;
    if (st) st->v0 = v3<double>(0., 0., 0.);
    return c;
  }
  LocalBody<double> la = local_body<double>(A, d3(0., 0., 0.), A.scaling);
  LocalBody<double> lb = local_body<double>(B, d3(0., 0., 0.), B.scaling);
  GjkResult<double> r = st ? gjk_sv_distance(la, lb, tol, *st) : gjk_sv_distance(la, lb, tol);
  if (st) st->v0 = r.v;
  *iters = r.iters;
  if (r.dist < kEpsilon) {
    c.status = 1;
    return c;
  }
  V3<double> ba = r.pa - r.pb;
  V3<double> pc = dv(r.pa, 2.) + dv(r.pb, 2.);
  double crust_sum = xadd(A.crust, B.crust);
  V3<double> ov = round3(dv(ba, r.dist));
  ov = sc(ov, crust_sum - r.dist);
  c.point = d3(pc.x, pc.y, pc.z);
  c.overlap_vector = d3(ov.x, ov.y, ov.z);
  c.overlap = r.dist - crust_sum;
  c.status = 0;
  return c;
}

// RigidBodyWithCrust::ClosestPoint_ErreurHandling (RigidBodyWithCrust.cpp:532-588):
// bodies shrunk by 'factor' crusts (scaling capped below at 0.5); the contact
// is imposed with overlap = -(crust sum) along the witness direction B->A.
// status 1 when even the shrunk bodies touch (fatal ContactError).
GG_HD ContactGeom convex_error_handling(const BodyRef& A, const BodyRef& B, const double ext_a[3],
                                        const double ext_b[3], double factor, double tol, bool accel = false) {
  double sa[3], sb[3];
  for (int i = 0; i < 3; ++i) {
    sa[i] = ext_a[i] < kEpsilon ? 1. : xdiv(xsub(ext_a[i], xmul(factor, A.crust)), ext_a[i]);
    sb[i] = ext_b[i] < kEpsilon ? 1. : xdiv(xsub(ext_b[i], xmul(factor, B.crust)), ext_b[i]);
    sa[i] = fmax(sa[i], 0.5);
    sb[i] = fmax(sb[i], 0.5);
  }
  LocalBody<double> la = local_body<double>(A, d3(0., 0., 0.), sa);
  LocalBody<double> lb = local_body<double>(B, d3(0., 0., 0.), sb);
  GjkStart<double> st;
  st.accel = accel;
  GjkResult<double> r = gjk_distance(la, lb, tol, st);
  ContactGeom c = no_contact();
  if (r.dist < kEpsilon) {
    c.status = 1;
    return c;
  }
  V3<double> ba = r.pa - r.pb;
  ba = dv(ba, norm(ba));
  V3<double> pc = dv(r.pa, 2.0) + dv(r.pb, 2.0);
  double imp = 1. * xadd(A.crust, B.crust);
  c.point = d3(pc.x, pc.y, pc.z);
  c.overlap_vector = d3(ba.x * imp, ba.y * imp, ba.z * imp);
  c.overlap = -imp;
  c.status = 0;
  return c;
}

}  // namespace gg
