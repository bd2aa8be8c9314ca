// contact_law.cuh -- Hooke, HookeMemory, Hertz and HertzMemory contact force
// models, templated on the arithmetic type (float for the mixed path, double
// for plain FP64).
//
//   HookeMemoryContactForceModel::performForcesCalculus  Component/src/HookeMemoryContactForceModel.cpp:72-193
//   HookeMemoryContactForceModel::computeTangentialVector :54-65
//   HookeContactForceModel::performForcesCalculus         Component/src/HookeContactForceModel.cpp:44-114
//   HertzContactForceModel::performForcesCalculus         Component/src/HertzContactForceModel.cpp:44-120
//   HertzMemoryContactForceModel::performForcesCalculus   Component/src/HertzMemoryContactForceModel.cpp:72-197
//
// The model always works from the point of view of body 0 (p0).  It returns
// the force on p0 (delFN + delFT, applied at the contact point) and the extra
// torque delM of rolling friction; p1 receives the exact negation
// (computeForces, HookeMemoryContactForceModel.cpp:200-249).
#pragma once

#include "../../include/grains_gpu.h"
#include "common.cuh"

namespace gg {

template <typename R>
struct LawParams {
  int type;  // GRAINS_GPU_HOOKE .. GRAINS_GPU_HERTZ_MEMORY, -1 = undefined pair
  int rolling;  // memory law with a rolling spring (mur != 0)
  R kn, en, etat, muc, kt, mur, etarpf, epst, kr, beta;
  R Es, Gs;     // Hertz laws: Young-like and shear moduli
  // the same parameters of the normal part in double, for the mixed path
  // (normal_part_fp64): kn, beta, etat, Es, Gs
  double kn64, beta64, etat64, Es64, Gs64;
};

// laws that keep a tangential (and rolling) spring per contact
GG_HD bool law_has_memory(int type) {
  return type == GRAINS_GPU_HOOKE_MEMORY || type == GRAINS_GPU_HERTZ_MEMORY;
}

// laws whose rolling torque delM is applied (m_kr / m_rolling_friction)
template <typename R>
GG_HD bool law_has_torque(const LawParams<R>& L) {
  return L.rolling || L.kr != R(0);
}

// Contact memory value of one pair seen from p0 (Component.hh:507-513)
template <typename R>
struct PairMemory {
  V3<R> kdelta, prev_normal, spring;
};

template <typename R>
struct BodyAtContact {
  V3<R> v;      // translational velocity
  V3<R> w;      // world angular velocity
  V3<R> lever;  // contact point - body centre
  V3<R> pos_minus_contact;  // centre - contact point (Hooke rolling term)
  R mass;
  R req;        // equivalent sphere radius (Component::getEquivalentSphereRadius)
};

template <typename R>
struct LawResult {
  V3<R> force;       // on p0
  V3<R> torque;      // extra torque on p0 (rolling), zero otherwise
  V3<R> tangential;  // the tangential part of `force` (delFT)
};

template <typename R>
GG_HD V3<R> velocity_at(const BodyAtContact<R>& b) {  // Particle.cpp:662-666
  return b.v + cross(b.w, b.lever);
}

// Branch flags of one law evaluation (optional output): which case of the
// tangential direction and whether Coulomb's limit was reached.  The law is
// smooth in its inputs between changes of these flags.
enum { kLawTangentVelocity = 1, kLawTangentSpring = 2, kLawSlip = 4 };

// computeTangentialVector (HookeMemoryContactForceModel.cpp:54-65)
template <typename R>
GG_HD V3<R> tangential_vector(R epst, R n_t, V3<R> ut, V3<R> kd, int* branch = nullptr) {
  if (norm(ut) > R(0.001)) {
    if (branch) *branch |= kLawTangentVelocity;
    return dv(-ut, norm(ut));
  }
  V3<R> s = kd + sc(ut, n_t);
  if ((norm(kd) > epst || norm(sc(ut, n_t)) > epst) && norm(s) > epst) {
    if (branch) *branch |= kLawTangentSpring;
    return dv(-s, norm(s));
  }
  return v3<R>(R(0), R(0), R(0));
}

// Tangential spring with memory, Coulomb slip and the rolling spring-dashpot,
// common to HookeMemory (HookeMemoryContactForceModel.cpp:140-192) and
// HertzMemory (HertzMemoryContactForceModel.cpp:129-192).  kt is the tangential
// stiffness, kn and gamman the normal stiffness and damping the rolling
// spring is built from (Jiang et al. 2005): constants for Hooke, functions of
// sqrt(Req deltan) for Hertz.  'existed' tells whether a memory entry was
// found; 'mem' holds it on entry (when existed) and the updated entry on exit.
template <typename R>
GG_HD LawResult<R> memory_tangent_rolling(const LawParams<R>& L, R dt, V3<R> normal, V3<R> v_t, V3<R> delFN,
                                          R normFN, R gammat, R kt, R kn, R gamman, const BodyAtContact<R>& b0,
                                          const BodyAtContact<R>& b1, bool existed, PairMemory<R>& mem,
                                          int* branch) {
  V3<R> viscousFT = sc(v_t, -gammat);
  Qt<R> qrot{v3<R>(R(0), R(0), R(0)), R(0)};
  if (existed) {
    qrot = q_rot_from_two(mem.prev_normal, normal);
    mem.kdelta = q_rotate(qrot, mem.kdelta);
  } else {
    mem.kdelta = v3<R>(R(0), R(0), R(0));
    mem.spring = v3<R>(R(0), R(0), R(0));
  }
  mem.kdelta = mem.kdelta + sc(v_t, dt * kt);
  mem.prev_normal = normal;
  V3<R> tij = tangential_vector(L.epst, gammat, v_t, mem.kdelta, branch);
  R normFT = norm(-mem.kdelta + viscousFT);
  V3<R> delFT;
  if (normFT <= L.muc * normFN) {
    delFT = sc(tij, norm(-mem.kdelta + viscousFT));
  } else {
    if (branch) *branch |= kLawSlip;
    // kt = 0 (HookeMemory without a spring) leaves the memory as it is
    if (kt != R(0)) mem.kdelta = dv(sc(tij, -L.muc * normFN) + viscousFT, kt);
    delFT = sc(tij, L.muc * normFN);
  }
  LawResult<R> out;
  out.force = delFN + delFT;
  out.tangential = delFT;
  out.torque = v3<R>(R(0), R(0), R(0));
  if (L.rolling) {
    R Req = R(1) / (R(1) / b0.req + R(1) / b1.req);
    R kr = R(3) * kn * L.mur * L.mur * Req * Req;
    R etar = R(3) * gamman * L.mur * L.mur * Req * Req;
    R max_normMk = L.mur * Req * normFN;
    V3<R> wrel = b0.w - b1.w;
    if (existed) mem.spring = q_rotate(qrot, mem.spring);
    mem.spring = mem.spring - sc(wrel, kr * dt);
    R normMk = norm(mem.spring);
    if (normMk > max_normMk) mem.spring = sc(mem.spring, max_normMk / normMk);
    out.torque = mem.spring - sc(wrel, L.etarpf * etar);
  }
  return out;
}

// Coulomb saturation of a purely viscous tangential force
// (HookeContactForceModel.cpp:86-96, HertzContactForceModel.cpp:91-101)
template <typename R>
GG_HD V3<R> coulomb_cap(V3<R> delFT, V3<R> v_t, R fn, int* branch) {
  R ft = norm(delFT);
  if (fn < ft) {
    if (branch) *branch |= kLawSlip;
    R nvt = norm(v_t);
    V3<R> tangent = v3<R>(R(0), R(0), R(0));
    if (nvt > R(kEpsilon)) tangent = dv(-v_t, nvt);
    delFT = sc(tangent, fn);
  }
  return delFT;
}

// Rolling resistance torque of the memoryless laws
// (HookeContactForceModel.cpp:99-111, HertzContactForceModel.cpp:104-117)
template <typename R>
GG_HD V3<R> kr_rolling_torque(R kr, R normFN, const BodyAtContact<R>& b0, const BodyAtContact<R>& b1) {
  V3<R> torque = v3<R>(R(0), R(0), R(0));
  if (kr != R(0)) {
    V3<R> wrel = b0.w - b1.w;
    R normwrel = norm(wrel);
    R normwtrel = norm(cross(b0.w, b0.pos_minus_contact) - cross(b1.w, b1.pos_minus_contact));
    if (normwrel > R(kEpsilon)) {
      R Req = R(1) / (R(1) / b0.req + R(1) / b1.req);
      torque = sc(wrel, -(kr * Req * normFN * normwtrel / normwrel));
    }
  }
  return torque;
}

// HookeMemory law
template <typename R>
GG_HD LawResult<R> hooke_memory(const LawParams<R>& L, R dt, V3<R> pen, const BodyAtContact<R>& b0,
                                const BodyAtContact<R>& b1, bool existed, PairMemory<R>& mem,
                                int* branch = nullptr) {
  V3<R> normal = round3(dv(pen, norm(pen)));
  V3<R> tmpV = velocity_at(b0) - velocity_at(b1);
  V3<R> v_n = sc(normal, dot(tmpV, normal));
  V3<R> v_t = tmpV - v_n;
  V3<R> delFN = sc(pen, L.kn);
  R avmass = R(1) / (R(1) / b0.mass + R(1) / b1.mass);
  R gamman = R(-2) * L.beta * gsqrt(avmass * L.kn);
  delFN = delFN - sc(v_n, gamman);
  R normFN = norm(delFN);
  R etat = L.etat == R(-1) ? -L.beta * gsqrt(L.kn / avmass) : L.etat;
  R gammat = R(2) * etat * avmass;
  return memory_tangent_rolling(L, dt, normal, v_t, delFN, normFN, gammat, L.kt, L.kn, gamman, b0, b1, existed,
                                mem, branch);
}

// Hooke law (no memory)
template <typename R>
GG_HD LawResult<R> hooke(const LawParams<R>& L, V3<R> pen, const BodyAtContact<R>& b0,
                         const BodyAtContact<R>& b1, int* branch = nullptr) {
  V3<R> normal = round3(dv(pen, norm(pen)));
  V3<R> tmpV = velocity_at(b0) - velocity_at(b1);
  V3<R> v_n = sc(normal, dot(tmpV, normal));
  V3<R> v_t = tmpV - v_n;
  V3<R> delFN = sc(pen, L.kn);
  R avmass = R(1) / (R(1) / b0.mass + R(1) / b1.mass);
  R gamman = R(-2) * L.beta * gsqrt(avmass * L.kn);
  delFN = delFN - sc(v_n, gamman);
  R normFN = norm(delFN);
  R etat = L.etat == R(-1) ? -L.beta * gsqrt(L.kn / avmass) : L.etat;
  R gammat = R(2) * etat * avmass;
  LawResult<R> out;
  out.tangential = coulomb_cap(sc(v_t, -gammat), v_t, L.muc * normFN, branch);
  out.force = delFN + out.tangential;
  out.torque = kr_rolling_torque(L.kr, normFN, b0, b1);
  return out;
}

// Normal part of both Hertz laws: stiffness (4/3) Es sqrt(Req deltan) and the
// damping -2 sqrt(5/6) beta sqrt(m* Sn), Sn = 2 Es sqrt(Req deltan); the
// tangential damping uses St = 8 Gs sqrt(Req deltan)
// (HertzContactForceModel.cpp:48-84).  deltan = -overlap distance > 0.
template <typename R>
struct HertzNormal {
  V3<R> normal, v_t, delFN;
  R normFN, kn, gamman, gammat, sqrtReqdeltan;
};

template <typename R>
GG_HD HertzNormal<R> hertz_normal(const LawParams<R>& L, V3<R> pen, R deltan, const BodyAtContact<R>& b0,
                                  const BodyAtContact<R>& b1) {
  HertzNormal<R> h;
  R Req = R(1) / (R(1) / b0.req + R(1) / b1.req);
  R avmass = R(1) / (R(1) / b0.mass + R(1) / b1.mass);
  h.sqrtReqdeltan = gsqrt(Req * deltan);
  R Sn = R(2) * L.Es * h.sqrtReqdeltan;
  R St = R(8) * L.Gs * h.sqrtReqdeltan;
  const R m2sqrt56 = R(-2. * 0.91287092917527690);  // -2 sqrt(5/6)
  h.normal = round3(dv(pen, norm(pen)));
  V3<R> tmpV = velocity_at(b0) - velocity_at(b1);
  V3<R> v_n = sc(h.normal, dot(tmpV, h.normal));
  h.v_t = tmpV - v_n;
  h.kn = R(4. / 3.) * L.Es * h.sqrtReqdeltan;
  h.delFN = sc(pen, h.kn);
  h.gamman = m2sqrt56 * L.beta * gsqrt(avmass * Sn);
  h.delFN = h.delFN - sc(v_n, h.gamman);
  h.normFN = norm(h.delFN);
  h.gammat = m2sqrt56 * L.beta * gsqrt(avmass * St);
  return h;
}

// Hertz law (no memory)
template <typename R>
GG_HD LawResult<R> hertz(const LawParams<R>& L, V3<R> pen, R deltan, const BodyAtContact<R>& b0,
                         const BodyAtContact<R>& b1, int* branch = nullptr) {
  const HertzNormal<R> h = hertz_normal(L, pen, deltan, b0, b1);
  LawResult<R> out;
  out.tangential = coulomb_cap(sc(h.v_t, -h.gammat), h.v_t, L.muc * h.normFN, branch);
  out.force = h.delFN + out.tangential;
  out.torque = kr_rolling_torque(L.kr, h.normFN, b0, b1);
  return out;
}

// HertzMemory law: tangential spring kt = 8 Gs sqrt(Req deltan)
// (HertzMemoryContactForceModel.cpp:141)
template <typename R>
GG_HD LawResult<R> hertz_memory(const LawParams<R>& L, R dt, V3<R> pen, R deltan, const BodyAtContact<R>& b0,
                                const BodyAtContact<R>& b1, bool existed, PairMemory<R>& mem,
                                int* branch = nullptr) {
  const HertzNormal<R> h = hertz_normal(L, pen, deltan, b0, b1);
  const R kt = R(8) * L.Gs * h.sqrtReqdeltan;
  return memory_tangent_rolling(L, dt, h.normal, h.v_t, h.delFN, h.normFN, h.gammat, kt, h.kn, h.gamman, b0, b1,
                                existed, mem, branch);
}

// ---- mixed precision: the normal part in double -----------------------------
// In FP32 the normal force kn * overlap - gamman * v_n loses its leading digits
// when the elastic and viscous terms nearly cancel (a contact about to open):
// relative errors of 1e-5 and more against FP64 on a settling bed.  The mixed
// path therefore forms the normal direction, the relative velocity at the
// contact point, its normal and tangential parts, the normal force and its
// norm, and the damping coefficients in double, from the double overlap
// vector, lever arms and masses and the FP32 velocities widened exactly.  The
// tangential spring, Coulomb's limit, the rolling terms, the contact memory and
// the force sums stay in FP32.  The double expressions follow the FP32 ones
// above term by term, so for R = double they would give the same bits.

// Double-precision inputs of one contact: the bodies' velocities and angular
// velocities, lever arms (contact point - centre), masses and equivalent
// radii.
struct PairFp64 {
  V3<double> v0, w0, lev0, v1, w1, lev1;
  double m0, m1, req0, req1;
};

// Normal part of a law evaluated in double, and its FP32 images for the rest.
template <typename R>
struct NormalFp64 {
  V3<double> delFN64;  // the normal force in double (for its torque)
  V3<R> normal, v_t, delFN;
  R normFN, kn, gamman, gammat;
  R kt;  // tangential stiffness: kt of HookeMemory, 8 Gs sqrt(Req deltan) of HertzMemory
};

template <typename R>
GG_HD NormalFp64<R> normal_part_fp64(const LawParams<R>& L, V3<double> pen, double deltan, const PairFp64& p) {
  const bool hertz = L.type == GRAINS_GPU_HERTZ || L.type == GRAINS_GPU_HERTZ_MEMORY;
  const V3<double> normal = round3(dv(pen, norm(pen)));
  const V3<double> tmpV = (p.v0 + cross(p.w0, p.lev0)) - (p.v1 + cross(p.w1, p.lev1));
  const V3<double> v_n = sc(normal, dot(tmpV, normal));
  const V3<double> v_t = tmpV - v_n;
  const double avmass = 1. / (1. / p.m0 + 1. / p.m1);
  double kn, gamman, gammat, kt = double(L.kt);
  if (hertz) {  // HertzContactForceModel.cpp:48-84, HertzMemoryContactForceModel.cpp:141
    const double Req = 1. / (1. / p.req0 + 1. / p.req1);
    const double sq = std::sqrt(Req * deltan);
    const double Sn = 2. * L.Es64 * sq, St = 8. * L.Gs64 * sq;
    const double m2sqrt56 = -2. * 0.91287092917527690;
    kn = (4. / 3.) * L.Es64 * sq;
    gamman = m2sqrt56 * L.beta64 * std::sqrt(avmass * Sn);
    gammat = m2sqrt56 * L.beta64 * std::sqrt(avmass * St);
    kt = St;
  } else {  // HookeMemoryContactForceModel.cpp:96-124, HookeContactForceModel.cpp:56-78
    kn = L.kn64;
    gamman = -2. * L.beta64 * std::sqrt(avmass * L.kn64);
    const double etat = L.etat64 == -1. ? -L.beta64 * std::sqrt(L.kn64 / avmass) : L.etat64;
    gammat = 2. * etat * avmass;
  }
  const V3<double> delFN = sc(pen, kn) - sc(v_n, gamman);
  NormalFp64<R> o;
  o.delFN64 = delFN;
  o.normal = v3<R>(R(normal.x), R(normal.y), R(normal.z));
  o.v_t = v3<R>(R(v_t.x), R(v_t.y), R(v_t.z));
  o.delFN = v3<R>(R(delFN.x), R(delFN.y), R(delFN.z));
  o.normFN = R(norm(delFN));
  o.kn = R(kn);
  o.gamman = R(gamman);
  o.gammat = R(gammat);
  o.kt = R(kt);
  return o;
}

// Any of the four laws with the normal part of normal_part_fp64 (mixed path).
template <typename R>
GG_HD LawResult<R> apply_contact_law_fp64_normal(const LawParams<R>& L, R dt, const NormalFp64<R>& nd,
                                                 const BodyAtContact<R>& b0, const BodyAtContact<R>& b1,
                                                 bool existed, PairMemory<R>& mem) {
  if (law_has_memory(L.type))
    return memory_tangent_rolling(L, dt, nd.normal, nd.v_t, nd.delFN, nd.normFN, nd.gammat, nd.kt, nd.kn, nd.gamman,
                                  b0, b1, existed, mem, (int*)nullptr);
  LawResult<R> out;
  out.tangential = coulomb_cap(sc(nd.v_t, -nd.gammat), nd.v_t, L.muc * nd.normFN, (int*)nullptr);
  out.force = nd.delFN + out.tangential;
  out.torque = kr_rolling_torque(L.kr, nd.normFN, b0, b1);
  return out;
}

// Any of the four laws.  deltan = -overlap distance (Hertz laws only).
template <typename R>
GG_HD LawResult<R> apply_contact_law(const LawParams<R>& L, R dt, V3<R> pen, R deltan, const BodyAtContact<R>& b0,
                                     const BodyAtContact<R>& b1, bool existed, PairMemory<R>& mem,
                                     int* branch = nullptr) {
  switch (L.type) {
    case GRAINS_GPU_HOOKE_MEMORY: return hooke_memory(L, dt, pen, b0, b1, existed, mem, branch);
    case GRAINS_GPU_HERTZ: return hertz(L, pen, deltan, b0, b1, branch);
    case GRAINS_GPU_HERTZ_MEMORY: return hertz_memory(L, dt, pen, deltan, b0, b1, existed, mem, branch);
    default: return hooke(L, pen, b0, b1, branch);
  }
}

}  // namespace gg
