// tangent_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle of the adjoint).
//
// A CPU FP64 restatement of the differentiable leapfrog run of the Grains3D
// DEM step for spheres with box walls, templated on the scalar so that it also
// runs on forward-mode dual numbers: it returns the final state and its
// derivatives along given directions of the initial velocities and of the
// contact-law parameters (kn, en, muc, kt).  The CUDA path's adjoint
// (grains_gpu_adjoint_*) is checked against these derivatives.
//
// The run (same as the CUDA path's differentiable run):
//   E_k: forces of the current state (k = 0..K), then
//   V += a_k F / m, W += a_k T / I (a_0 = dt/2, a_k = dt, final half kick),
//   X += dt V (k < K); kdelta and rolling springs zeroed after E_0
// restating Grains::Simulation (Base/src/Grains.cpp:169-174, 344-364),
// SecondOrderLeapFrog::Move / advanceVelocity (TimeIntegration/src/
// SecondOrderLeapFrog.cpp:44-95; for spheres the body-frame SSP-RK3 reduces to
// W += a T / I), the broadphase as a set (Base/src/LinkedCell.cpp:1019-1103),
// ClosestPointSPHERESPHERE / SPHEREBOX (Geometry/src/RigidBodyWithCrust.cpp:
// 596-721, Box.cpp:466-768), HookeMemory (Component/src/
// HookeMemoryContactForceModel.cpp:54-249) and Hooke (Component/src/
// HookeContactForceModel.cpp:44-163), contact memory (Component/src/
// Component.cpp:570-689).  Contact pairs are owned by the lower index.
// Compiled with -ffp-contract=off: the double run rounds like the CUDA FP64 run.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <utility>
#include <vector>

namespace {

constexpr double EPS = 1.e-10;  // Basic.hh EPSILON
constexpr double PI = 3.14159265358979323846;
constexpr int LANES = 8;

struct Dual {
  double v;
  double d[LANES];
  Dual() : v(0.) { std::memset(d, 0, sizeof(d)); }
  Dual(double x) : v(x) { std::memset(d, 0, sizeof(d)); }  // NOLINT: implicit constants
};
inline Dual operator+(const Dual& a, const Dual& b) {
  Dual r(a.v + b.v);
  for (int l = 0; l < LANES; ++l) r.d[l] = a.d[l] + b.d[l];
  return r;
}
inline Dual operator-(const Dual& a, const Dual& b) {
  Dual r(a.v - b.v);
  for (int l = 0; l < LANES; ++l) r.d[l] = a.d[l] - b.d[l];
  return r;
}
inline Dual operator-(const Dual& a) {
  Dual r(-a.v);
  for (int l = 0; l < LANES; ++l) r.d[l] = -a.d[l];
  return r;
}
inline Dual operator*(const Dual& a, const Dual& b) {
  Dual r(a.v * b.v);
  for (int l = 0; l < LANES; ++l) r.d[l] = a.d[l] * b.v + a.v * b.d[l];
  return r;
}
inline Dual operator/(const Dual& a, const Dual& b) {
  Dual r(a.v / b.v);
  for (int l = 0; l < LANES; ++l) r.d[l] = (a.d[l] - r.v * b.d[l]) / b.v;
  return r;
}
inline Dual sqrt_(const Dual& a) {
  Dual r(std::sqrt(a.v));
  for (int l = 0; l < LANES; ++l) r.d[l] = r.v > 0. ? a.d[l] / (2. * r.v) : 0.;
  return r;
}
inline Dual log_(const Dual& a) {
  Dual r(std::log(a.v));
  for (int l = 0; l < LANES; ++l) r.d[l] = a.d[l] / a.v;
  return r;
}
inline double sqrt_(double a) { return std::sqrt(a); }
inline double log_(double a) { return std::log(a); }
inline double val(double a) { return a; }
inline double val(const Dual& a) { return a.v; }

template <typename S>
struct V {
  S x, y, z;
};
template <typename S>
V<S> mk(S a, S b, S c) {
  return V<S>{a, b, c};
}
template <typename S>
V<S> operator+(const V<S>& a, const V<S>& b) {
  return mk<S>(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename S>
V<S> operator-(const V<S>& a, const V<S>& b) {
  return mk<S>(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename S>
V<S> operator-(const V<S>& a) {
  return mk<S>(-a.x, -a.y, -a.z);
}
template <typename S>
V<S> sc(const V<S>& a, const S& d) {
  return mk<S>(a.x * d, a.y * d, a.z * d);
}
template <typename S>
V<S> dv(const V<S>& a, const S& d) {
  return mk<S>(a.x / d, a.y / d, a.z / d);
}
template <typename S>
S dot(const V<S>& a, const V<S>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename S>
V<S> cross(const V<S>& a, const V<S>& b) {  // Vector3::operator^, Vector3.cpp:114-119
  return mk<S>(a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x);
}
template <typename S>
S norm(const V<S>& a) {
  return sqrt_(a.x * a.x + a.y * a.y + a.z * a.z);
}
template <typename S>
V<S> round3(const V<S>& a) {  // Group3::round, Group3.cpp:390-395
  return mk<S>(std::fabs(val(a.x)) < EPS ? S(0.) : a.x, std::fabs(val(a.y)) < EPS ? S(0.) : a.y,
               std::fabs(val(a.z)) < EPS ? S(0.) : a.z);
}
template <typename S>
V<S> cst(const double* p) {
  return mk<S>(S(p[0]), S(p[1]), S(p[2]));
}

// quaternions: Quaternion::setRotFromTwoVectors (:263-289), rotateVector (:293-298)
template <typename S>
struct Q {
  V<S> v;
  S w;
};
template <typename S>
Q<S> rot_from_two(const V<S>& u, const V<S>& v) {
  S nn = sqrt_(dot(u, u) * dot(v, v));
  S real = nn + dot(u, v);
  V<S> vect;
  if (val(real) < 1.e-6 * val(nn)) {
    real = S(0.);
    vect = std::fabs(val(u.x)) > std::fabs(val(u.z)) ? mk<S>(-u.y, u.x, S(0.)) : mk<S>(S(0.), -u.z, u.y);
  } else {
    vect = cross(u, v);
  }
  S s = S(1.) / sqrt_(vect.x * vect.x + vect.y * vect.y + vect.z * vect.z + real * real);
  return Q<S>{sc(vect, s), s * real};
}
template <typename S>
V<S> rotate(const Q<S>& q, const V<S>& v) {
  S nv = norm(q.v);
  return (sc(v, q.w * q.w - nv * nv) + sc(q.v, S(2.) * dot(v, q.v))) + sc(cross(q.v, v), S(2.) * q.w);
}

struct LawP {
  int type = -1;  // 0 Hooke, 1 HookeMemory
  double kn = 0, en = 0, etat = -1, muc = 0, kt = 0, mur = 0, etarpf = 0, epst = 0, kr = 0;
};

template <typename S>
struct Mem {
  V<S> kd, n, sp;
};

template <typename S>
struct Body {  // a body at the contact point
  V<S> v, w, lever, pmc;
  double mass, req;
};

template <typename S>
struct LawS {
  int type, rolling;
  S kn, beta, etat, muc, kt, mur, etarpf, epst, kr;
};

// HookeMemoryContactForceModel::computeTangentialVector (:54-65)
template <typename S>
V<S> tangential(const S& epst, const S& nt, const V<S>& ut, const V<S>& kd) {
  if (val(norm(ut)) > 0.001) return dv(-ut, norm(ut));
  V<S> s = kd + sc(ut, nt);
  if ((val(norm(kd)) > val(epst) || val(norm(sc(ut, nt))) > val(epst)) && val(norm(s)) > val(epst))
    return dv(-s, norm(s));
  return mk<S>(S(0.), S(0.), S(0.));
}

template <typename S>
V<S> vel_at(const Body<S>& b) {
  return b.v + cross(b.w, b.lever);
}

// force on p0 and rolling torque on p0; memory updated (HookeMemory) in place
template <typename S>
void law(const LawS<S>& L, double dt, const V<S>& pen, const Body<S>& b0, const Body<S>& b1, bool existed,
         Mem<S>& m, V<S>& force, V<S>& torque) {
  V<S> normal = round3(dv(pen, norm(pen)));
  V<S> tmpV = vel_at(b0) - vel_at(b1);
  V<S> v_n = sc(normal, dot(tmpV, normal));
  V<S> v_t = tmpV - v_n;
  V<S> delFN = sc(pen, L.kn);
  S avmass = S(1.) / (S(1.) / S(b0.mass) + S(1.) / S(b1.mass));
  S gamman = S(-2.) * L.beta * sqrt_(avmass * L.kn);
  delFN = delFN - sc(v_n, gamman);
  S normFN = norm(delFN);
  S etat = val(L.etat) == -1. ? -L.beta * sqrt_(L.kn / avmass) : L.etat;
  S gammat = S(2.) * etat * avmass;
  torque = mk<S>(S(0.), S(0.), S(0.));
  if (L.type == 1) {
    V<S> viscousFT = sc(v_t, -gammat);
    Q<S> qrot{mk<S>(S(0.), S(0.), S(0.)), S(0.)};
    if (existed) {
      qrot = rot_from_two(m.n, normal);
      m.kd = rotate(qrot, m.kd);
    } else {
      m.kd = mk<S>(S(0.), S(0.), S(0.));
      m.sp = mk<S>(S(0.), S(0.), S(0.));
    }
    m.kd = m.kd + sc(v_t, S(dt) * L.kt);
    m.n = normal;
    V<S> tij = tangential(L.epst, gammat, v_t, m.kd);
    S normFT = norm(-m.kd + viscousFT);
    V<S> delFT;
    if (val(normFT) <= val(L.muc * normFN)) {
      delFT = sc(tij, norm(-m.kd + viscousFT));
    } else {
      if (val(L.kt) != 0.) m.kd = dv(sc(tij, -L.muc * normFN) + viscousFT, L.kt);
      delFT = sc(tij, L.muc * normFN);
    }
    force = delFN + delFT;
    if (L.rolling) {
      S Req = S(1.) / (S(1.) / S(b0.req) + S(1.) / S(b1.req));
      S kr = S(3.) * L.kn * L.mur * L.mur * Req * Req;
      S etar = S(3.) * gamman * L.mur * L.mur * Req * Req;
      S max_normMk = L.mur * Req * normFN;
      V<S> wrel = b0.w - b1.w;
      if (existed) m.sp = rotate(qrot, m.sp);
      m.sp = m.sp - sc(wrel, kr * S(dt));
      S normMk = norm(m.sp);
      if (val(normMk) > val(max_normMk)) m.sp = sc(m.sp, max_normMk / normMk);
      torque = m.sp - sc(wrel, L.etarpf * etar);
    }
  } else {
    V<S> delFT = sc(v_t, -gammat);
    S fn = L.muc * normFN;
    S ft = norm(delFT);
    if (val(fn) < val(ft)) {
      S nvt = norm(v_t);
      V<S> tangent = mk<S>(S(0.), S(0.), S(0.));
      if (val(nvt) > EPS) tangent = dv(-v_t, nvt);
      delFT = sc(tangent, fn);
    }
    force = delFN + delFT;
    if (val(L.kr) != 0.) {
      V<S> wrel = b0.w - b1.w;
      S normwrel = norm(wrel);
      S normwtrel = norm(cross(b0.w, b0.pmc) - cross(b1.w, b1.pmc));
      if (val(normwrel) > EPS) {
        S Req = S(1.) / (S(1.) / S(b0.req) + S(1.) / S(b1.req));
        torque = sc(wrel, -(L.kr * Req * normFN * normwtrel / normwrel));
      }
    }
  }
}

struct Wall {
  double b[9], o[3], e[3];  // basis (row major), origin, half edges
  double crust;
  int material;
  double bbc[3], bbe[3];
  double req;
};

struct Setup {
  int n;
  const double *radius, *mass, *inertia, *crust;
  const int* material;
  double origin[3], size[3], cell, g[3];
  int nbi, nbj, nbk;
  double ex, ey, ez;
  std::vector<Wall> walls;
  int n_mat;
  std::vector<LawP> laws;
};

// box corner helpers of Box::IntersectionPointSPHERE in the box frame
// (sphere_box in the CUDA path; Box.cpp:466-768)
template <typename S>
bool sphere_box(const Wall& W, const V<S>& c, double r, double crust_sum, V<S>& point, V<S>& pen, S& ov_out,
                bool& error) {
  error = false;
  // local = B^T c - B^T o (Transform::setToInverseTransform + operator())
  double bt[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) bt[3 * i + j] = W.b[3 * j + i];
  double io[3];
  for (int i = 0; i < 3; ++i) io[i] = -((bt[3 * i] * W.o[0] + bt[3 * i + 1] * W.o[1]) + bt[3 * i + 2] * W.o[2]);
  V<S> g;
  g.x = ((S(bt[0]) * c.x + S(bt[1]) * c.y) + S(bt[2]) * c.z) + S(io[0]);
  g.y = ((S(bt[3]) * c.x + S(bt[4]) * c.y) + S(bt[5]) * c.z) + S(io[1]);
  g.z = ((S(bt[6]) * c.x + S(bt[7]) * c.y) + S(bt[8]) * c.z) + S(io[2]);
  const double e[3] = {W.e[0], W.e[1], W.e[2]};
  int s[3];
  const double gv[3] = {val(g.x), val(g.y), val(g.z)};
  for (int a = 0; a < 3; ++a) s[a] = gv[a] > e[a] ? 1 : (gv[a] < -e[a] ? -1 : 0);
  const int nz = (s[0] != 0) + (s[1] != 0) + (s[2] != 0);
  if (nz == 0) {
    error = true;
    return false;
  }
  V<S> cp = g;
  S ov;
  S* gc[3] = {&g.x, &g.y, &g.z};
  S* cc[3] = {&cp.x, &cp.y, &cp.z};
  if (nz == 1) {
    const int a = s[0] ? 0 : (s[1] ? 1 : 2);
    S nd = s[a] > 0 ? *gc[a] - S(e[a]) : S(-e[a]) - *gc[a];
    if (!(val(nd) < r)) return false;
    ov = nd - S(r);
    *cc[a] = s[a] > 0 ? S(e[a]) + S(0.5) * ov : S(-e[a]) - S(0.5) * ov;
  } else {
    V<S> d;
    d.x = s[0] ? g.x - S(s[0] * e[0]) : S(0.);
    d.y = s[1] ? g.y - S(s[1] * e[1]) : S(0.);
    d.z = s[2] ? g.z - S(s[2] * e[2]) : S(0.);
    S nd = norm(d);
    if (!(val(nd) < r)) return false;
    ov = nd - S(r);
    cp = g - sc(d, S(1.) + (S(0.5) * ov) / nd);
  }
  if (-val(ov) >= crust_sum) {
    error = true;
    return false;
  }
  point.x = ((S(W.b[0]) * cp.x + S(W.b[1]) * cp.y) + S(W.b[2]) * cp.z) + S(W.o[0]);
  point.y = ((S(W.b[3]) * cp.x + S(W.b[4]) * cp.y) + S(W.b[5]) * cp.z) + S(W.o[1]);
  point.z = ((S(W.b[6]) * cp.x + S(W.b[7]) * cp.y) + S(W.b[8]) * cp.z) + S(W.o[2]);
  V<S> ab = point - c;
  pen = sc(ab, ov / norm(ab));
  ov_out = ov;
  return true;
}

// one contact seen from its owner o (lower index, or the particle for a wall)
template <typename S>
struct ContactS {
  V<S> force, torque, lever0, lever1;
};

template <typename S>
struct Run {
  const Setup& su;
  std::vector<V<S>> X, Vv, W;
  std::vector<LawS<S>> laws;  // per law slot (n_mat x n_mat)
  std::map<std::pair<int, int>, Mem<S>> mem, next;
  double dt = 0.;
  explicit Run(const Setup& s) : su(s) {}

  void cell_of(const V<S>& x, int id[3]) const {
    id[0] = int(std::floor((val(x.x) - su.origin[0]) / su.ex));
    id[1] = int(std::floor((val(x.y) - su.origin[1]) / su.ey));
    id[2] = int(std::floor((val(x.z) - su.origin[2]) / su.ez));
  }

  // contacts of particle i: overlapping spheres (sorted by index), then walls
  void partners(int i, const std::vector<std::vector<int>>& cells, std::vector<int>& out) const {
    out.clear();
    int id[3];
    cell_of(X[i], id);
    for (int a = 0; a < 3; ++a) id[a] = std::min(std::max(id[a], 0), (a == 0 ? su.nbi : a == 1 ? su.nbj : su.nbk) - 1);
    for (int dj = -1; dj <= 1; ++dj)
      for (int dk = -1; dk <= 1; ++dk)
        for (int di = -1; di <= 1; ++di) {
          int ci = id[0] + di, cj = id[1] + dj, ck = id[2] + dk;
          if (ci < 0 || cj < 0 || ck < 0 || ci >= su.nbi || cj >= su.nbj || ck >= su.nbk) continue;
          for (int p : cells[cj * su.nbk * su.nbi + ck * su.nbi + ci]) {
            if (p == i) continue;
            V<double> ab = mk(val(X[p].x) - val(X[i].x), val(X[p].y) - val(X[i].y), val(X[p].z) - val(X[i].z));
            if (std::sqrt(ab.x * ab.x + ab.y * ab.y + ab.z * ab.z) - (su.radius[i] + su.radius[p]) < 0.) out.push_back(p);
          }
        }
    std::sort(out.begin(), out.end());
    for (size_t w = 0; w < su.walls.size(); ++w) {
      const Wall& Wl = su.walls[w];
      const double r = su.radius[i];
      bool in = true;
      const double p[3] = {val(X[i].x), val(X[i].y), val(X[i].z)};
      for (int a = 0; a < 3; ++a) in = in && std::fabs(Wl.bbc[a] - p[a]) <= Wl.bbe[a] + r;
      if (!in) continue;
      V<S> pt, pen;
      S ov;
      bool err;
      if (sphere_box(Wl, X[i], r, su.crust[i] + Wl.crust, pt, pen, ov, err)) out.push_back(-(int)w - 1);
      if (err) throw std::runtime_error("contact error");
    }
  }

  bool contact(int o, int code, ContactS<S>& c, int& slot, std::pair<int, int>& key) {
    Body<S> b0, b1;
    V<S> pen, point;
    const double r0 = su.radius[o];
    b0.v = Vv[o];
    b0.w = W[o];
    b0.mass = su.mass[o];
    b0.req = r0;
    const V<S> A = X[o];
    V<S> B;
    if (code >= 0) {
      const int p = code;
      B = X[p];
      V<S> ab = B - A;
      S nab = norm(ab);
      S dist = nab - S(r0 + su.radius[p]);
      if (!(val(dist) < 0.)) return false;
      if (-val(dist) >= su.crust[o] + su.crust[p]) throw std::runtime_error("contact error");
      point = A + dv(sc(ab, S(r0) + S(0.5) * dist), nab);
      pen = sc(dv(ab, nab), dist);
      b1.v = Vv[p];
      b1.w = W[p];
      b1.mass = su.mass[p];
      b1.req = su.radius[p];
      slot = su.material[o] * su.n_mat + su.material[p];
    } else {
      const Wall& Wl = su.walls[-code - 1];
      S ov;
      bool err;
      if (!sphere_box(Wl, A, r0, su.crust[o] + Wl.crust, point, pen, ov, err)) return false;
      B = cst<S>(Wl.o);
      b1.v = mk<S>(S(0.), S(0.), S(0.));
      b1.w = mk<S>(S(0.), S(0.), S(0.));
      b1.mass = 1.e20;
      b1.req = Wl.req;
      slot = su.material[o] * su.n_mat + Wl.material;
    }
    b0.lever = point - A;
    b0.pmc = A - point;
    b1.lever = point - B;
    b1.pmc = B - point;
    const LawS<S>& L = laws[slot];
    key = std::make_pair(o, code);
    Mem<S> m;
    m.kd = m.n = m.sp = mk<S>(S(0.), S(0.), S(0.));
    bool existed = false;
    if (L.type == 1) {
      auto it = mem.find(key);
      if (it != mem.end()) {
        m = it->second;
        existed = true;
      }
    }
    law(L, dt, pen, b0, b1, existed, m, c.force, c.torque);
    c.lever0 = b0.lever;
    c.lever1 = b1.lever;
    if (L.type == 1) next[key] = m;
    return true;
  }
};

}  // namespace

namespace {

template <typename S>
void run_steps(Run<S>& R, int K, double dt) {
  const Setup& su = R.su;
  const int n = su.n;
  R.dt = dt;
  std::vector<std::vector<int>> cells((size_t)su.nbi * su.nbj * su.nbk);
  std::vector<int> list;
  std::vector<V<S>> F(n), T(n);
  for (int k = 0; k <= K; ++k) {
    for (auto& c : cells) c.clear();
    for (int i = 0; i < n; ++i) {
      int id[3];
      R.cell_of(R.X[i], id);
      if (id[0] < 0 || id[1] < 0 || id[2] < 0 || id[0] >= su.nbi || id[1] >= su.nbj || id[2] >= su.nbk)
        throw std::runtime_error("particle outside the grid");
      cells[(size_t)id[1] * su.nbk * su.nbi + (size_t)id[2] * su.nbi + id[0]].push_back(i);
    }
    R.next.clear();
    for (int i = 0; i < n; ++i) {
      F[i] = mk<S>(S(su.g[0] * su.mass[i]), S(su.g[1] * su.mass[i]), S(su.g[2] * su.mass[i]));
      T[i] = mk<S>(S(0.), S(0.), S(0.));
      R.partners(i, cells, list);
      for (int code : list) {
        const bool own = code < 0 || i < code;
        const int o = own ? i : code, pc = own ? code : i;
        ContactS<S> c;
        int slot;
        std::pair<int, int> key;
        if (!R.contact(o, pc, c, slot, key)) continue;
        const V<S> f = own ? c.force : -c.force;
        F[i] = F[i] + f;
        T[i] = T[i] + cross(own ? c.lever0 : c.lever1, f);
        const LawS<S>& L = R.laws[slot];
        if (L.rolling || val(L.kr) != 0.) T[i] = T[i] + (own ? c.torque : -c.torque);
      }
    }
    if (k == 0)
      for (auto& kv : R.next) kv.second.kd = kv.second.sp = mk<S>(S(0.), S(0.), S(0.));
    R.mem.swap(R.next);
    const double h1 = 0.5 * dt, h2 = (k == 0 || k == K) ? 0. : 0.5 * dt;
    for (int i = 0; i < n; ++i) {
      const V<S> acc = dv(F[i], S(su.mass[i] * 1.));
      const V<S> alpha = dv(T[i], S(1. * su.inertia[i]));
      R.Vv[i] = R.Vv[i] + sc(acc, S(h1));
      R.W[i] = R.W[i] + sc(alpha, S(h1));
      if (h2 != 0.) {
        R.Vv[i] = R.Vv[i] + sc(acc, S(h2));
        R.W[i] = R.W[i] + sc(alpha, S(h2));
      }
      if (k < K) R.X[i] = R.X[i] + sc(R.Vv[i], S(dt));
    }
  }
}

template <typename S>
LawS<S> make_law(const LawP& p, const double* seeds /* 4 per lane or null */, int lanes, int stride);

template <>
LawS<double> make_law<double>(const LawP& p, const double*, int, int) {
  LawS<double> L;
  L.type = p.type;
  L.rolling = p.type == 1 && p.mur != 0.;
  L.kn = p.kn;
  L.beta = std::log(p.en) / std::sqrt(PI * PI + std::log(p.en) * std::log(p.en));
  L.etat = p.etat;
  L.muc = p.muc;
  L.kt = p.kt;
  L.mur = p.mur;
  L.etarpf = p.etarpf;
  L.epst = p.epst;
  L.kr = p.kr;
  return L;
}

template <>
LawS<Dual> make_law<Dual>(const LawP& p, const double* seeds, int lanes, int stride) {
  LawS<Dual> L;
  L.type = p.type;
  L.rolling = p.type == 1 && p.mur != 0.;
  Dual kn(p.kn), en(p.en), muc(p.muc), kt(p.kt);
  for (int l = 0; l < lanes && seeds; ++l) {
    kn.d[l] = seeds[l * stride + 0];
    en.d[l] = seeds[l * stride + 1];
    muc.d[l] = seeds[l * stride + 2];
    kt.d[l] = seeds[l * stride + 3];
  }
  L.kn = kn;
  const Dual le = log_(en);
  L.beta = le / sqrt_(Dual(PI * PI) + le * le);
  L.beta.v = std::log(p.en) / std::sqrt(PI * PI + std::log(p.en) * std::log(p.en));
  L.etat = Dual(p.etat);
  L.muc = muc;
  L.kt = kt;
  L.mur = Dual(p.mur);
  L.etarpf = Dual(p.etarpf);
  L.epst = Dual(p.epst);
  L.kr = Dual(p.kr);
  return L;
}

}  // namespace

// Runs n_steps of the differentiable leapfrog from (x0, v0, w0) and writes the
// final state; with n_dirs > 0 also the derivatives of the final state along
// n_dirs directions, each a perturbation of the initial velocities (3n) and of
// (kn, en, muc, kt) of every law slot (n_mat^2 x 4).  Returns 0, or 1 on a
// contact / motion error.
//   domain: origin[3], size[3], cell_size, gravity[3]
//   walls: per wall 12 doubles of transform (row-major basis, origin), 3 half
//          edges, crust, material, equivalent radius (18 doubles)
//   laws: per slot (a * n_mat + b) type, kn, en, etat, muc, kt, mur, etarpf,
//         epst, kr (10 doubles; type < 0 = undefined)
extern "C" int grains_tangent_run(int n, const double* x0, const double* v0, const double* w0,
                                  const double* radius, const double* mass, const double* inertia,
                                  const double* crust, const int* material, const double* domain, int n_walls,
                                  const double* walls, int n_mat, const double* laws, int n_steps, double dt,
                                  int n_dirs, const double* dir_v0, const double* dir_laws, double* x, double* v,
                                  double* w, double* tx, double* tv, double* tw) {
  Setup su;
  su.n = n;
  su.radius = radius;
  su.mass = mass;
  su.inertia = inertia;
  su.crust = crust;
  su.material = material;
  for (int a = 0; a < 3; ++a) {
    su.origin[a] = domain[a];
    su.size[a] = domain[3 + a];
    su.g[a] = domain[7 + a];
  }
  su.cell = domain[6];
  int nb[3];
  for (int a = 0; a < 3; ++a) nb[a] = std::max(int((su.size[a] + EPS) / su.cell), 1);  // LinkedCell::set, :47-140
  su.nbi = nb[0];
  su.nbj = nb[1];
  su.nbk = nb[2];
  su.ex = su.size[0] / nb[0];
  su.ey = su.size[1] / nb[1];
  su.ez = su.size[2] / nb[2];
  for (int k = 0; k < n_walls; ++k) {
    const double* p = walls + 18 * k;
    Wall W;
    for (int t = 0; t < 9; ++t) W.b[t] = p[t];
    for (int t = 0; t < 3; ++t) W.o[t] = p[9 + t];
    for (int t = 0; t < 3; ++t) W.e[t] = p[12 + t];
    W.crust = p[15];
    W.material = (int)p[16];
    W.req = p[17];
    for (int a = 0; a < 3; ++a) {
      W.bbc[a] = W.o[a];
      W.bbe[a] = std::fabs(W.b[3 * a]) * W.e[0] + std::fabs(W.b[3 * a + 1]) * W.e[1] + std::fabs(W.b[3 * a + 2]) * W.e[2];
    }
    su.walls.push_back(W);
  }
  su.n_mat = n_mat;
  su.laws.resize((size_t)n_mat * n_mat);
  for (int k = 0; k < n_mat * n_mat; ++k) {
    const double* p = laws + 10 * k;
    LawP L;
    L.type = (int)p[0];
    L.kn = p[1];
    L.en = p[2];
    L.etat = p[3];
    L.muc = p[4];
    L.kt = p[5];
    L.mur = p[6];
    L.etarpf = p[7];
    L.epst = p[8];
    L.kr = p[9];
    su.laws[k] = L;
  }
  try {
    if (n_dirs <= 0) {
      Run<double> R(su);
      R.X.resize(n);
      R.Vv.resize(n);
      R.W.resize(n);
      for (int i = 0; i < n; ++i) {
        R.X[i] = mk(x0[3 * i], x0[3 * i + 1], x0[3 * i + 2]);
        R.Vv[i] = mk(v0[3 * i], v0[3 * i + 1], v0[3 * i + 2]);
        R.W[i] = mk(w0[3 * i], w0[3 * i + 1], w0[3 * i + 2]);
      }
      for (auto& L : su.laws) R.laws.push_back(make_law<double>(L, nullptr, 0, 0));
      run_steps(R, n_steps, dt);
      for (int i = 0; i < n; ++i) {
        const double a[3] = {R.X[i].x, R.X[i].y, R.X[i].z}, b[3] = {R.Vv[i].x, R.Vv[i].y, R.Vv[i].z},
                     c[3] = {R.W[i].x, R.W[i].y, R.W[i].z};
        for (int t = 0; t < 3; ++t) {
          x[3 * i + t] = a[t];
          v[3 * i + t] = b[t];
          w[3 * i + t] = c[t];
        }
      }
      return 0;
    }
    const int nslot = n_mat * n_mat;
    for (int d0 = 0; d0 < n_dirs; d0 += LANES) {
      const int lanes = std::min(LANES, n_dirs - d0);
      Run<Dual> R(su);
      R.X.resize(n);
      R.Vv.resize(n);
      R.W.resize(n);
      for (int i = 0; i < n; ++i) {
        R.X[i] = mk(Dual(x0[3 * i]), Dual(x0[3 * i + 1]), Dual(x0[3 * i + 2]));
        Dual vv[3] = {Dual(v0[3 * i]), Dual(v0[3 * i + 1]), Dual(v0[3 * i + 2])};
        for (int l = 0; l < lanes; ++l)
          for (int t = 0; t < 3; ++t) vv[t].d[l] = dir_v0 ? dir_v0[(size_t)(d0 + l) * 3 * n + 3 * i + t] : 0.;
        R.Vv[i] = mk(vv[0], vv[1], vv[2]);
        R.W[i] = mk(Dual(w0[3 * i]), Dual(w0[3 * i + 1]), Dual(w0[3 * i + 2]));
      }
      std::vector<double> seeds((size_t)lanes * 4);
      for (int k = 0; k < nslot; ++k) {
        for (int l = 0; l < lanes; ++l)
          for (int t = 0; t < 4; ++t) seeds[4 * l + t] = dir_laws ? dir_laws[((size_t)(d0 + l) * nslot + k) * 4 + t] : 0.;
        R.laws.push_back(make_law<Dual>(su.laws[k], seeds.data(), lanes, 4));
      }
      run_steps(R, n_steps, dt);
      for (int i = 0; i < n; ++i) {
        const Dual* a[3] = {&R.X[i].x, &R.X[i].y, &R.X[i].z};
        const Dual* b[3] = {&R.Vv[i].x, &R.Vv[i].y, &R.Vv[i].z};
        const Dual* c[3] = {&R.W[i].x, &R.W[i].y, &R.W[i].z};
        for (int t = 0; t < 3; ++t) {
          if (d0 == 0) {
            x[3 * i + t] = a[t]->v;
            v[3 * i + t] = b[t]->v;
            w[3 * i + t] = c[t]->v;
          }
          for (int l = 0; l < lanes; ++l) {
            const size_t o = (size_t)(d0 + l) * 3 * n + 3 * i + t;
            tx[o] = a[t]->d[l];
            tv[o] = b[t]->d[l];
            tw[o] = c[t]->d[l];
          }
        }
      }
    }
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}
