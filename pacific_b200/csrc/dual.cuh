// dual.cuh -- forward-mode dual numbers with L tangent lanes, for the adjoint
// of the DEM step.  The adjoint kernels evaluate the contact geometry and the
// contact law of one contact with Dual<R, L> inputs seeded on L of its inputs,
// which yields L columns of the contact's local Jacobian in one pass; the
// adjoint (a vector-Jacobian product) is contracted from them.  The value part
// of every operation is the plain R operation in the same order, so the
// primal values (and every branch taken by the law) equal those of the R
// evaluation in the step kernels.
#pragma once

#include "common.cuh"

namespace gg {

template <typename T, int L>
struct Dual {
  T v;
  T d[L];
  GG_HD Dual() : v(T(0)) {
#pragma unroll
    for (int l = 0; l < L; ++l) d[l] = T(0);
  }
  GG_HD explicit Dual(double x) : v(T(x)) {
#pragma unroll
    for (int l = 0; l < L; ++l) d[l] = T(0);
  }
  GG_HD explicit Dual(float x) : v(T(x)) {
#pragma unroll
    for (int l = 0; l < L; ++l) d[l] = T(0);
  }
  GG_HD explicit Dual(int x) : v(T(x)) {
#pragma unroll
    for (int l = 0; l < L; ++l) d[l] = T(0);
  }
};

template <typename T, int L>
GG_HD Dual<T, L> seeded(T v, int lane) {  // value v, tangent e_lane (lane outside [0, L): constant)
  Dual<T, L> r;
  r.v = v;
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = (l == lane) ? T(1) : T(0);
  return r;
}

template <typename T, int L>
GG_HD Dual<T, L> operator+(const Dual<T, L>& a, const Dual<T, L>& b) {
  Dual<T, L> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = a.d[l] + b.d[l];
  return r;
}
template <typename T, int L>
GG_HD Dual<T, L> operator-(const Dual<T, L>& a, const Dual<T, L>& b) {
  Dual<T, L> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = a.d[l] - b.d[l];
  return r;
}
template <typename T, int L>
GG_HD Dual<T, L> operator-(const Dual<T, L>& a) {
  Dual<T, L> r;
  r.v = -a.v;
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = -a.d[l];
  return r;
}
template <typename T, int L>
GG_HD Dual<T, L> operator*(const Dual<T, L>& a, const Dual<T, L>& b) {
  Dual<T, L> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = a.d[l] * b.v + a.v * b.d[l];
  return r;
}
template <typename T, int L>
GG_HD Dual<T, L> operator/(const Dual<T, L>& a, const Dual<T, L>& b) {
  Dual<T, L> r;
  r.v = a.v / b.v;
  const T inv = T(1) / b.v;
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = (a.d[l] - r.v * b.d[l]) * inv;
  return r;
}
template <typename T, int L>
GG_HD Dual<T, L> gsqrt(const Dual<T, L>& a) {
  Dual<T, L> r;
  r.v = std::sqrt(a.v);
  const T h = r.v > T(0) ? T(0.5) / r.v : T(0);
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = a.d[l] * h;
  return r;
}
template <typename T, int L>
GG_HD Dual<T, L> gabs(const Dual<T, L>& a) {
  return a.v < T(0) ? -a : a;
}

// comparisons act on the values
template <typename T, int L>
GG_HD bool operator<(const Dual<T, L>& a, const Dual<T, L>& b) {
  return a.v < b.v;
}
template <typename T, int L>
GG_HD bool operator>(const Dual<T, L>& a, const Dual<T, L>& b) {
  return a.v > b.v;
}
template <typename T, int L>
GG_HD bool operator<=(const Dual<T, L>& a, const Dual<T, L>& b) {
  return a.v <= b.v;
}
template <typename T, int L>
GG_HD bool operator>=(const Dual<T, L>& a, const Dual<T, L>& b) {
  return a.v >= b.v;
}
template <typename T, int L>
GG_HD bool operator==(const Dual<T, L>& a, const Dual<T, L>& b) {
  return a.v == b.v;
}
template <typename T, int L>
GG_HD bool operator!=(const Dual<T, L>& a, const Dual<T, L>& b) {
  return a.v != b.v;
}

// sum over lanes of the tangent of each component of x weighted by w
template <typename T, int L>
GG_HD void accumulate_vjp(const V3<Dual<T, L>>& x, V3<T> w, T out[L]) {
#pragma unroll
  for (int l = 0; l < L; ++l) out[l] += w.x * x.x.d[l] + w.y * x.y.d[l] + w.z * x.z.d[l];
}

}  // namespace gg
