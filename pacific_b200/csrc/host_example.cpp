// host_example.cpp -- a C++ caller of the DEM step through the reference-style
// adaptor of grains_gpu.hpp: 125 spheres dropped in a closed box, 2000 KDK
// steps on the device, then the reference's MotionError raised by a particle
// thrown faster than its crust allows.  Prints one JSON line.
#include <cstdio>
#include <vector>

#include "../../include/grains_gpu.hpp"

using namespace grains_gpu;

static void walls(LinkedCellGPU& lc, const double lo[3], const double hi[3], double crust) {
  std::vector<grains_gpu_obstacle> obs;
  const double t = 0.5e-3;
  for (int axis = 0; axis < 3; ++axis)
    for (int upper = 0; upper < 2; ++upper) {
      double e[3], c[3];
      for (int k = 0; k < 3; ++k) {
        e[k] = hi[k] - lo[k] + 2 * t;
        c[k] = 0.5 * (lo[k] + hi[k]);
      }
      e[axis] = t;
      c[axis] = upper ? hi[axis] + t / 2 : lo[axis] - t / 2;
      grains_gpu_obstacle o{};
      o.id = -1 - (int)obs.size();
      o.shape = lc.addShape(Box(e[0], e[1], e[2]));
      o.material = 1;
      o.crust = crust;
      double tr[12] = {1, 0, 0, 0, 1, 0, 0, 0, 1, c[0], c[1], c[2]};
      for (int k = 0; k < 12; ++k) o.transform[k] = tr[k];
      obs.push_back(o);
    }
  lc.LinkObstacles(obs);
}

int main() {
  const double r = 1e-3, crust = 5e-5, rho = 2500., dt = 1e-5;
  const double lo[3] = {0, 0, 0}, hi[3] = {12e-3, 12e-3, 24e-3}, size[3] = {12e-3, 12e-3, 24e-3};
  const double g[3] = {0, 0, -9.81};
  LinkedCellGPU lc(125, GRAINS_GPU_MIXED);
  lc.set(lo, size, 2 * r, g);
  Sphere sph(r);
  int sid = lc.addShape(sph);
  HookeMemoryContactForceModel law(1e5, 0.9, 0.5, 0.8e5);
  lc.setContactForceModel(0, 0, law);
  lc.setContactForceModel(0, 1, law);
  walls(lc, lo, hi, crust);
  ParticleSet ps;
  for (int k = 0; k < 125; ++k) {
    double x[3] = {1.2e-3 + 2.4e-3 * (k % 5), 1.2e-3 + 2.4e-3 * ((k / 5) % 5), 1.2e-3 + 2.4e-3 * (k / 25)};
    ps.add(k, sid, sph, rho, 0, crust, x);
  }
  lc.Link(&ps);
  lc.initializeLeapFrog(0., dt);
  double t = lc.Simulation(2000, 0., dt);
  lc.download(&ps);
  double zmin = 1, zmax = 0;
  int coord = 0;
  for (size_t i = 0; i < ps.size(); ++i) {
    zmin = std::min(zmin, ps.position[3 * i + 2]);
    zmax = std::max(zmax, ps.position[3 * i + 2]);
    coord += ps.coordination[i];
  }
  // a particle thrown at 10 m/s moves 0.1 mm in one step: more than its 0.05 mm crust
  bool motion_error = false;
  ps.velocity[3 * 60 + 2] = 10.;
  grains_gpu_particles v = ps.view();
  check(grains_gpu_update_particles(lc.context(), &v), lc.context());
  try {
    lc.Simulation(1, t, dt);
  } catch (MotionError&) {
    motion_error = true;
  }
  std::printf("{\"time\": %.9g, \"zmin\": %.9g, \"zmax\": %.9g, \"contacts\": %d, \"motion_error\": %s}\n", t, zmin,
              zmax, coord, motion_error ? "true" : "false");
  return 0;
}
