// Host build of the library's narrowphase (pacific_b200/csrc/gjk.cuh): the
// signed-volume GJK against Johnson's GJK and against closed forms, on seeded
// random pairs of boxes, cylinders and octahedra near contact.  Compiled and
// run by tests/test_gjk_cpu.py; prints a summary line and exits 1 on failure.
#include <cstdio>
#include <random>

#include "../pacific_b200/csrc/gjk.cuh"

using namespace gg;

static M3 random_rotation(std::mt19937_64& g) {
  std::normal_distribution<double> N;
  double q[4], s = 0;
  for (double& x : q) {
    x = N(g);
    s += x * x;
  }
  s = std::sqrt(s);
  const double x = q[0] / s, y = q[1] / s, z = q[2] / s, w = q[3] / s;
  M3 m;
  m.m[0] = 1 - 2 * (y * y + z * z); m.m[1] = 2 * (x * y - z * w); m.m[2] = 2 * (x * z + y * w);
  m.m[3] = 2 * (x * y + z * w); m.m[4] = 1 - 2 * (x * x + z * z); m.m[5] = 2 * (y * z - x * w);
  m.m[6] = 2 * (x * z - y * w); m.m[7] = 2 * (y * z + x * w); m.m[8] = 1 - 2 * (x * x + y * y);
  return m;
}

static double octahedron[18] = {1.2e-3, 0, 0, -1.2e-3, 0, 0, 0, 1.2e-3, 0, 0, -1.2e-3, 0, 0, 0, 1.2e-3, 0, 0, -1.2e-3};

static BodyRef body(int type, M3 basis, D3 origin) {
  BodyRef r;
  r.type = type;
  r.nverts = 6;
  r.verts = octahedron;
  r.radius = type == 0 ? 1e-3 : (type == 1 ? std::sqrt(3.) * 1e-3 : (type == 2 ? std::sqrt(2.) * 1e-3 : 1.2e-3));
  r.cyl_r = 1e-3;
  r.cyl_hh = 1e-3;
  r.ext = d3(1e-3, 1e-3, 1e-3);
  r.crust = 5e-5;
  r.basis = basis;
  r.origin = origin;
  for (int i = 0; i < 3; ++i) r.scaling[i] = 1.;
  return r;
}

int main() {
  int failures = 0;
  // closed forms: axis-aligned boxes a gap apart, spheres
  M3 id;
  for (int t = 0; t < 9; ++t) id.m[t] = (t % 4 == 0) ? 1. : 0.;
  for (double gap : {1e-6, 3e-5, 2e-4}) {
    BodyRef a = body(1, id, d3(0, 0, 0)), b = body(1, id, d3(2e-3 + gap, 3e-4, -2e-4));
    LocalBody<double> la = local_body<double>(a, d3(0, 0, 0), a.scaling);
    LocalBody<double> lb = local_body<double>(b, d3(0, 0, 0), b.scaling);
    const GjkResult<double> r = gjk_sv_distance(la, lb, 1e-10);
    if (std::fabs(r.dist - gap) > 1e-15) {
      std::printf("box gap %g: distance %.17g\n", gap, r.dist);
      ++failures;
    }
    BodyRef s1 = body(0, id, d3(0, 0, 0)), s2 = body(0, id, d3(0.6 * (2e-3 + gap), 0.8 * (2e-3 + gap), 0.));
    LocalBody<double> l1 = local_body<double>(s1, d3(0, 0, 0), s1.scaling);
    LocalBody<double> l2 = local_body<double>(s2, d3(0, 0, 0), s2.scaling);
    const GjkResult<double> q = gjk_sv_distance(l1, l2, 1e-10);
    const double exact = gap;
    if (std::fabs(q.dist - exact) > 1e-10 * exact + 1e-16) {
      std::printf("spheres gap %g: distance %.17g, exact %.17g\n", gap, q.dist, exact);
      ++failures;
    }
  }
  // random convex pairs.  GjkResult::lower is a certified lower bound of the
  // distance (the largest support-plane separation met), and the distance is
  // that of a point of the Minkowski difference, an upper bound: the
  // signed-volume answer must lie within the tolerance above the best lower
  // bound either algorithm certified.
  std::mt19937_64 g(11);
  std::uniform_real_distribution<double> U(-1, 1);
  int pairs = 0, capped = 0;
  double worst = -1.;
  for (int t = 0; t < 40000; ++t) {
    const BodyRef a = body(1 + (int)(g() % 3), random_rotation(g), d3(0, 0, 0));
    const BodyRef b = body(1 + (int)(g() % 3), random_rotation(g),
                           d3(2.4e-3 + 1e-3 * U(g), 1e-3 * U(g), 1e-3 * U(g)));
    LocalBody<double> la = local_body<double>(a, d3(0, 0, 0), a.scaling);
    LocalBody<double> lb = local_body<double>(b, d3(0, 0, 0), b.scaling);
    const GjkResult<double> sv = gjk_sv_distance(la, lb, 1e-10);
    const GjkResult<double> jo = gjk_distance(la, lb, 1e-10);
    if (sv.iters >= 1000) ++capped;
    if (sv.dist < 1e-7) continue;  // touching: the crust handles these
    ++pairs;
    // the stopping test is relative (1e-10) or absolute (1e-14 m); where
    // rounding stalls the iteration on curved bodies (a support point the
    // sub-algorithm drops), up to a few 1e-13 m remain (Johnson's GJK ends
    // in its backup procedure on the same pairs, 1e-11 m away)
    const double lower = std::fmax(sv.lower, jo.lower);
    const double excess = (sv.dist - lower) - (2e-10 * sv.dist + 5e-13);
    if (excess > worst) worst = excess;
    // the witness points are the distance apart
    const double wd = norm(sv.pa - sv.pb);
    if (std::fabs(wd - sv.dist) > 1e-12 * sv.dist + 1e-17) ++failures;
  }
  if (worst > 0.) ++failures;
  if (capped) ++failures;
  std::printf("pairs %d worst_excess_over_tolerance %.3g iteration_cap_hits %d failures %d\n", pairs, worst, capped,
              failures);
  return failures ? 1 : 0;
}
