// contact_law.cuh -- Hooke and HookeMemory contact force models, templated on
// the arithmetic type (float for the mixed path, double for plain FP64).
//
//   HookeMemoryContactForceModel::performForcesCalculus  Component/src/HookeMemoryContactForceModel.cpp:72-193
//   HookeMemoryContactForceModel::computeTangentialVector :54-65
//   HookeContactForceModel::performForcesCalculus         Component/src/HookeContactForceModel.cpp:44-114
//
// The model always works from the point of view of body 0 (p0).  It returns
// the force on p0 (delFN + delFT, applied at the contact point) and the extra
// torque delM of rolling friction; p1 receives the exact negation
// (computeForces, HookeMemoryContactForceModel.cpp:200-249).
#pragma once

#include "common.cuh"

namespace gg {

template <typename R>
struct LawParams {
  int type;  // GRAINS_GPU_HOOKE / GRAINS_GPU_HOOKE_MEMORY, -1 = undefined pair
  int rolling;
  R kn, en, etat, muc, kt, mur, etarpf, epst, kr, beta;
};

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
  V3<R> force;  // on p0
  V3<R> torque; // extra torque on p0 (rolling), zero otherwise
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

// HookeMemory law.  'existed' tells whether a memory entry was found; 'mem'
// holds it on entry (when existed) and the updated entry on exit.
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
  V3<R> viscousFT = sc(v_t, -gammat);
  Qt<R> qrot{v3<R>(R(0), R(0), R(0)), R(0)};
  if (existed) {
    qrot = q_rot_from_two(mem.prev_normal, normal);
    mem.kdelta = q_rotate(qrot, mem.kdelta);
  } else {
    mem.kdelta = v3<R>(R(0), R(0), R(0));
    mem.spring = v3<R>(R(0), R(0), R(0));
  }
  mem.kdelta = mem.kdelta + sc(v_t, dt * L.kt);
  mem.prev_normal = normal;
  V3<R> tij = tangential_vector(L.epst, gammat, v_t, mem.kdelta, branch);
  R normFT = norm(-mem.kdelta + viscousFT);
  V3<R> delFT;
  if (normFT <= L.muc * normFN) {
    delFT = sc(tij, norm(-mem.kdelta + viscousFT));
  } else {
    if (branch) *branch |= kLawSlip;
    if (L.kt != R(0)) mem.kdelta = dv(sc(tij, -L.muc * normFN) + viscousFT, L.kt);
    delFT = sc(tij, L.muc * normFN);
  }
  LawResult<R> out;
  out.force = delFN + delFT;
  out.torque = v3<R>(R(0), R(0), R(0));
  if (L.rolling) {
    R Req = R(1) / (R(1) / b0.req + R(1) / b1.req);
    R kr = R(3) * L.kn * L.mur * L.mur * Req * Req;
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
  V3<R> delFT = sc(v_t, -gammat);
  R fn = L.muc * normFN;
  R ft = norm(delFT);
  if (fn < ft) {
    if (branch) *branch |= kLawSlip;
    R nvt = norm(v_t);
    V3<R> tangent = v3<R>(R(0), R(0), R(0));
    if (nvt > R(kEpsilon)) tangent = dv(-v_t, nvt);
    delFT = sc(tangent, fn);
  }
  LawResult<R> out;
  out.force = delFN + delFT;
  out.torque = v3<R>(R(0), R(0), R(0));
  if (L.kr != R(0)) {
    V3<R> wrel = b0.w - b1.w;
    R normwrel = norm(wrel);
    R normwtrel = norm(cross(b0.w, b0.pos_minus_contact) - cross(b1.w, b1.pos_minus_contact));
    if (normwrel > R(kEpsilon)) {
      R Req = R(1) / (R(1) / b0.req + R(1) / b1.req);
      out.torque = sc(wrel, -(L.kr * Req * normFN * normwtrel / normwrel));
    }
  }
  return out;
}

}  // namespace gg
