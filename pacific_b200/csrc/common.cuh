// common.cuh -- small vector algebra shared by host set-up code and sm_100a
// kernels of the Grains3D DEM step.
//
// Two kinds of arithmetic live here:
//  * "exact" double helpers (xadd, xmul, ...) that always round each
//    operation separately (__dadd_rn & co. on the device, plain IEEE
//    operations on the x86-64 host, which has no contraction without
//    -march flags).  They are used wherever a decision must reproduce the
//    reference's double-precision result bit for bit: cell binning
//    (Cell::GetCell, Base/src/Cell.cpp:172-184), overlap distances
//    (RigidBodyWithCrust.cpp:596-721) and the obstacle prefilter
//    (BBox::InZone, Geometry/src/BBox.cpp:166-185).
//  * generic templated vectors V3<R> for R = float (mixed precision) or
//    double (plain FP64) used by the contact law and the integrator.
//
// Expression orders follow the reference's Group3 / Vector3 / Quaternion
// operators (Geometry/src/Group3.cpp:149-330, Vector3.cpp:114-160,
// Quaternion.cpp:95-460) so the plain FP64 path rounds like the reference.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define GG_HD __host__ __device__ __forceinline__
#else
#define GG_HD inline
#endif

namespace gg {

constexpr double kEpsilon = 1.e-10;   // Base/include/Basic.hh:26
constexpr double kEpsilon2 = 1.e-15;  // Basic.hh:27
constexpr double kEpsilon3 = 1.e-20;  // Basic.hh:28
constexpr double kPi = 3.14159265358979323846;
constexpr double kObstacleMass = 1.e20;  // Component/src/Component.cpp:16

// ---- exact-rounding double operations -------------------------------------
GG_HD double xadd(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
GG_HD double xsub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
GG_HD double xmul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
GG_HD double xdiv(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
GG_HD double xsqrt(double a) {
#if defined(__CUDA_ARCH__)
  return __dsqrt_rn(a);
#else
  return std::sqrt(a);
#endif
}

struct D3 {
  double x, y, z;
};
GG_HD D3 d3(double a, double b, double c) { return D3{a, b, c}; }
GG_HD D3 xsub3(D3 a, D3 b) { return d3(xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z)); }
GG_HD D3 xadd3(D3 a, D3 b) { return d3(xadd(a.x, b.x), xadd(a.y, b.y), xadd(a.z, b.z)); }
GG_HD D3 xscale(D3 a, double s) { return d3(xmul(a.x, s), xmul(a.y, s), xmul(a.z, s)); }
GG_HD D3 xdivs(D3 a, double s) { return d3(xdiv(a.x, s), xdiv(a.y, s), xdiv(a.z, s)); }
GG_HD double xdot(D3 a, D3 b) { return xadd(xadd(xmul(a.x, b.x), xmul(a.y, b.y)), xmul(a.z, b.z)); }
GG_HD double xnorm(D3 a) { return xsqrt(xdot(a, a)); }
GG_HD double xget(D3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// ---- generic scalar functions -------------------------------------------------
// Unqualified gsqrt / gabs in the generic code below let a forward-mode dual
// number (dual.cuh) overload them; for float and double they are std::sqrt
// and std::fabs.
template <typename R>
GG_HD R gsqrt(R x) {
  return std::sqrt(x);
}
template <typename R>
GG_HD R gabs(R x) {
  return std::fabs(x);
}

// ---- generic vectors -------------------------------------------------------
template <typename R>
struct V3 {
  R x, y, z;
};
template <typename R>
GG_HD V3<R> v3(R a, R b, R c) {
  return V3<R>{a, b, c};
}
template <typename R>
GG_HD V3<R> operator+(V3<R> a, V3<R> b) {
  return v3<R>(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename R>
GG_HD V3<R> operator-(V3<R> a, V3<R> b) {
  return v3<R>(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename R>
GG_HD V3<R> operator-(V3<R> a) {
  return v3<R>(-a.x, -a.y, -a.z);
}
template <typename R>
GG_HD V3<R> sc(V3<R> a, R d) {  // Group3 * d and d * Group3: g[i] * d
  return v3<R>(a.x * d, a.y * d, a.z * d);
}
template <typename R>
GG_HD V3<R> dv(V3<R> a, R d) {
  return v3<R>(a.x / d, a.y / d, a.z / d);
}
template <typename R>
GG_HD R dot(V3<R> a, V3<R> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename R>
GG_HD V3<R> cross(V3<R> a, V3<R> b) {  // Vector3::operator^, Vector3.cpp:114-119
  return v3<R>(a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x);
}
template <typename R>
GG_HD R norm(V3<R> a) {
  return gsqrt(a.x * a.x + a.y * a.y + a.z * a.z);
}
template <typename R>
GG_HD R norm2(V3<R> a) {
  return a.x * a.x + a.y * a.y + a.z * a.z;
}
template <typename R>
GG_HD V3<R> round3(V3<R> a) {  // Group3::round(EPSILON), Group3.cpp:390-395
  const R tol = R(kEpsilon);
  return v3<R>(gabs(a.x) < tol ? R(0) : a.x, gabs(a.y) < tol ? R(0) : a.y, gabs(a.z) < tol ? R(0) : a.z);
}
template <typename R>
GG_HD V3<R> from_d3(D3 a) {
  return v3<R>(R(a.x), R(a.y), R(a.z));
}
template <typename R>
GG_HD D3 to_d3(V3<R> a) {
  return d3(double(a.x), double(a.y), double(a.z));
}

// ---- quaternions (vector part v, scalar w) ----------------------------------
template <typename R>
struct Qt {
  V3<R> v;
  R w;
};
template <typename R>
GG_HD Qt<R> qconj(Qt<R> q) {
  return Qt<R>{-q.v, q.w};
}
template <typename R>
GG_HD Qt<R> qmul(Qt<R> a, Qt<R> b) {  // Quaternion::operator*, Quaternion.cpp:442-448
  R t = (a.w * b.w) - dot(a.v, b.v);
  V3<R> vt = (cross(a.v, b.v) + sc(b.v, a.w)) + sc(a.v, b.w);
  return Qt<R>{vt, t};
}
template <typename R>
GG_HD Qt<R> qmult_left_vec(Qt<R> q, V3<R> lhs) {  // [0,lhs] x q, Quaternion.cpp:95-100
  R t = dot(-lhs, q.v);
  V3<R> vt = cross(lhs, q.v) + sc(lhs, q.w);
  return Qt<R>{vt, t};
}
template <typename R>
GG_HD V3<R> qmult_to_v3(Qt<R> a, Qt<R> rhs) {  // Quaternion::multToVector3, :108-113
  return (cross(a.v, rhs.v) + sc(rhs.v, a.w)) + sc(a.v, rhs.w);
}
template <typename R>
GG_HD R qnorm(Qt<R> q) {
  return gsqrt(q.v.x * q.v.x + q.v.y * q.v.y + q.v.z * q.v.z + q.w * q.w);
}
// q x [0,v] x conj(q) written as the reference composes it in
// ParticleKinematics::Move (ParticleKinematics.cpp:79-80): q.multToVector3((v, conj(q)))
template <typename R>
GG_HD V3<R> q_to_world(Qt<R> q, V3<R> v) {
  return qmult_to_v3(q, qmult_left_vec(qconj(q), v));
}
// conj(q) x [0,v] x q (ParticleKinematics.cpp:66-67)
template <typename R>
GG_HD V3<R> q_to_body(Qt<R> q, V3<R> v) {
  return qmult_to_v3(qconj(q), qmult_left_vec(q, v));
}
// Quaternion::setRotFromTwoVectors, Quaternion.cpp:263-289
template <typename R>
GG_HD Qt<R> q_rot_from_two(V3<R> u, V3<R> v) {
  R nn = gsqrt(dot(u, u) * dot(v, v));
  R real = nn + dot(u, v);
  V3<R> vect;
  if (real < R(1.e-6) * nn) {
    real = R(0);
    vect = gabs(u.x) > gabs(u.z) ? v3<R>(-u.y, u.x, R(0)) : v3<R>(R(0), -u.z, u.y);
  } else {
    vect = cross(u, v);
  }
  Qt<R> qq{vect, real};
  R s = R(1) / qnorm(qq);
  return Qt<R>{sc(qq.v, s), s * qq.w};
}
// Quaternion::rotateVector, Quaternion.cpp:293-298
template <typename R>
GG_HD V3<R> q_rotate(Qt<R> q, V3<R> v) {
  R nv = norm(q.v);
  return (sc(v, q.w * q.w - nv * nv) + sc(q.v, R(2) * dot(v, q.v))) + sc(cross(q.v, v), R(2) * q.w);
}

// ---- 3x3 matrices (row major) ----------------------------------------------
struct M3 {
  double m[9];
};
GG_HD D3 mrow(const M3& a, int i) { return d3(a.m[3 * i], a.m[3 * i + 1], a.m[3 * i + 2]); }
// Transform::operator(): basis * p + origin, exact rounding (Transform.cpp:312-317)
GG_HD D3 xapply(const M3& b, D3 o, D3 p) {
  return d3(xadd(xdot(mrow(b, 0), p), o.x), xadd(xdot(mrow(b, 1), p), o.y), xadd(xdot(mrow(b, 2), p), o.z));
}
// v * M, Matrix::tdot (Matrix.cpp:238-241, 527-530)
GG_HD D3 xvecmat(D3 v, const M3& a) {
  D3 r;
  r.x = xadd(xadd(xmul(a.m[0], v.x), xmul(a.m[3], v.y)), xmul(a.m[6], v.z));
  r.y = xadd(xadd(xmul(a.m[1], v.x), xmul(a.m[4], v.y)), xmul(a.m[7], v.z));
  r.z = xadd(xadd(xmul(a.m[2], v.x), xmul(a.m[5], v.y)), xmul(a.m[8], v.z));
  return r;
}
GG_HD M3 mtranspose(const M3& a) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[3 * i + j] = a.m[3 * j + i];
  return r;
}
// Transform::composeWithScaling -> Matrix::multiplyByScalingMatrix (Matrix.cpp:347-358)
GG_HD M3 mscale_cols(const M3& a, double sx, double sy, double sz) {
  M3 r = a;
  for (int i = 0; i < 3; ++i) {
    r.m[3 * i] = xmul(r.m[3 * i], sx);
    r.m[3 * i + 1] = xmul(r.m[3 * i + 1], sy);
    r.m[3 * i + 2] = xmul(r.m[3 * i + 2], sz);
  }
  return r;
}
// Transform::composeLeftByRotation, Transform.cpp:140-157 (plain arithmetic;
// the FP64 kernels are built without contraction)
GG_HD void mrotate_left(M3& mm, Qt<double> q) {
  double qx = q.v.x, qy = q.v.y, qz = q.v.z, qw = q.w;
  M3 s = mm;
  for (int i = 0; i < 3; ++i) {
    double px = qy * s.m[6 + i] - qz * s.m[3 + i] + qw * s.m[i];
    double py = qz * s.m[i] - qx * s.m[6 + i] + qw * s.m[3 + i];
    double pz = qx * s.m[3 + i] - qy * s.m[i] + qw * s.m[6 + i];
    double pw = -qx * s.m[i] - qy * s.m[3 + i] - qz * s.m[6 + i];
    mm.m[i] = qy * pz - qz * py - pw * qx + qw * px;
    mm.m[3 + i] = qz * px - qx * pz - pw * qy + qw * py;
    mm.m[6 + i] = qx * py - qy * px - pw * qz + qw * pz;
  }
}

}  // namespace gg
