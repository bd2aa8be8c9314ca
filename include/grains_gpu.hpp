// grains_gpu.hpp -- header-only C++ host adaptor over the C ABI of
// grains_gpu.h, mirroring the interfaces of the reference Grains3D that the
// DEM step plugs into:
//
//   Convex (Geometry/include/Convex.hh:88-123)      -> grains_gpu::Convex, Sphere, Box, Cylinder, Polyhedron
//   ContactForceModel (Component/include/ContactForceModel.hh:43-68)
//                                                    -> grains_gpu::ContactForceModel, HookeContactForceModel,
//                                                       HookeMemoryContactForceModel, HertzContactForceModel,
//                                                       HertzMemoryContactForceModel
//   App / AppCollision (Base/include/App.hh:38-39, AppCollision.hh:79-100)
//                                                    -> grains_gpu::App, AppCollision, LinkedCellGPU
//   TimeIntegrator::Move / advanceVelocity (TimeIntegration/include/TimeIntegrator.hh:47-66)
//                                                    -> LinkedCellGPU::Move / advanceVelocity
//   ContactError / MotionError / SimulationError (Base/include/Error.hh:19,75,129)
//
// The adaptor owns the device context; particles are described by the
// ParticleSet structure of arrays (the host image of AllComponents' active
// particles).  Errors reported by the device are rethrown as the reference's
// exception classes so a time loop written against the reference behaves the
// same (Grains.cpp:423-450).
#ifndef GRAINS_GPU_HPP
#define GRAINS_GPU_HPP

#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "grains_gpu.h"

namespace grains_gpu {

// ---- exceptions (Error.hh) ---------------------------------------------------
struct GrainsError : std::runtime_error {
  int code;
  GrainsError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
struct ContactError : GrainsError {
  using GrainsError::GrainsError;
};
struct MotionError : GrainsError {
  using GrainsError::GrainsError;
};
struct SimulationError : GrainsError {
  using GrainsError::GrainsError;
};

inline void check(int rc, const grains_gpu_ctx* ctx) {
  if (rc == GRAINS_GPU_OK) return;
  char buf[1024] = {0};
  if (ctx) grains_gpu_last_error(ctx, buf, sizeof(buf));
  std::string m = std::string(buf) + " (status " + std::to_string(rc) + ")";
  if (rc & GRAINS_GPU_CONTACT_ERROR) throw ContactError(rc, m);
  if (rc & GRAINS_GPU_MOTION_ERROR) throw MotionError(rc, m);
  if (rc & GRAINS_GPU_OUT_OF_GRID) throw SimulationError(rc, m);
  throw GrainsError(rc, m);
}

// ---- convex shapes (metadata uploaded once per context) -----------------------
enum ConvexType { SPHERE = GRAINS_GPU_SPHERE, BOX = GRAINS_GPU_BOX, CYLINDER = GRAINS_GPU_CYLINDER,
                  POLYHEDRON = GRAINS_GPU_POLYHEDRON };

class Convex {
 public:
  virtual ~Convex() = default;
  virtual ConvexType getConvexType() const = 0;
  virtual std::vector<double> params() const = 0;
  double getVolume() const { return props().volume; }
  double computeCircumscribedRadius() const { return props().circ; }
  // principal inertia per unit density; inertia_1 = its inverse (Convex::BuildInertia)
  bool BuildInertia(double* inertia, double* inertia_1) const {
    Props p = props();
    for (int i = 0; i < 6; ++i) inertia[i] = inertia_1[i] = 0.;
    inertia[0] = p.inertia[0];
    inertia[3] = p.inertia[1];
    inertia[5] = p.inertia[2];
    inertia_1[0] = 1. / inertia[0];
    inertia_1[3] = 1. / inertia[3];
    inertia_1[5] = 1. / inertia[5];
    return true;
  }

 private:
  struct Props {
    double volume, circ, inertia[3];
  };
  Props props() const {
    Props p{};
    std::vector<double> v = params();
    check(grains_gpu_shape_properties(getConvexType(), v.data(), (int32_t)v.size(), &p.volume, &p.circ,
                                      p.inertia),
          nullptr);
    return p;
  }
};

class Sphere : public Convex {
 public:
  explicit Sphere(double r) : r_(r) {}
  ConvexType getConvexType() const override { return SPHERE; }
  std::vector<double> params() const override { return {r_}; }
  double getRadius() const { return r_; }

 private:
  double r_;
};

class Box : public Convex {  // full edge lengths, like Box(double x, double y, double z)
 public:
  Box(double lx, double ly, double lz) : l_{lx, ly, lz} {}
  ConvexType getConvexType() const override { return BOX; }
  std::vector<double> params() const override { return {l_[0], l_[1], l_[2]}; }

 private:
  double l_[3];
};

class Cylinder : public Convex {  // axis = local Y (Cylinder.cpp:112-133)
 public:
  Cylinder(double r, double h) : r_(r), h_(h) {}
  ConvexType getConvexType() const override { return CYLINDER; }
  std::vector<double> params() const override { return {r_, h_}; }

 private:
  double r_, h_;
};

class Polyhedron : public Convex {
 public:
  Polyhedron(std::vector<double> xyz, std::vector<std::vector<int>> faces) : v_(std::move(xyz)), f_(std::move(faces)) {}
  ConvexType getConvexType() const override { return POLYHEDRON; }
  std::vector<double> params() const override {
    std::vector<double> p;
    p.push_back(double(v_.size() / 3));
    p.insert(p.end(), v_.begin(), v_.end());
    p.push_back(double(f_.size()));
    for (auto& f : f_) {
      p.push_back(double(f.size()));
      for (int i : f) p.push_back(double(i));
    }
    return p;
  }

 private:
  std::vector<double> v_;
  std::vector<std::vector<int>> f_;
};

// ---- contact force models ----------------------------------------------------
class ContactForceModel {
 public:
  virtual ~ContactForceModel() = default;
  virtual std::string name() const = 0;
  virtual int law() const = 0;
  virtual std::vector<double> parameters() const = 0;
};

// HookeContactForceModel (HookeContactForceModel.cpp:9-18, 170-199)
class HookeContactForceModel : public ContactForceModel {
 public:
  HookeContactForceModel(double kn, double en, double muc, double kr, double etat = -1.)
      : kn_(kn), en_(en), etat_(etat), muc_(muc), kr_(kr) {}
  std::string name() const override { return "HookeContactForceModel"; }
  int law() const override { return GRAINS_GPU_HOOKE; }
  std::vector<double> parameters() const override { return {kn_, en_, etat_, muc_, kr_}; }

 private:
  double kn_, en_, etat_, muc_, kr_;
};

// HookeMemoryContactForceModel (HookeMemoryContactForceModel.cpp:11-29, 256-308)
class HookeMemoryContactForceModel : public ContactForceModel {
 public:
  HookeMemoryContactForceModel(double kn, double en, double muc, double kt, double etat = -1., double mur = 0.,
                               double etarpf = 0., double epst = 0.)
      : p_{kn, en, etat, muc, kt, mur, etarpf, epst} {}
  std::string name() const override { return "HookeMemoryContactForceModel"; }
  int law() const override { return GRAINS_GPU_HOOKE_MEMORY; }
  std::vector<double> parameters() const override { return std::vector<double>(p_, p_ + 8); }

 private:
  double p_[8];
};

// HertzContactForceModel (HertzContactForceModel.cpp:12-21, 236-276); Gs
// defaults to Es / 4 as when the XML omits it
class HertzContactForceModel : public ContactForceModel {
 public:
  HertzContactForceModel(double Es, double en, double muc, double kr, double Gs = -1.)
      : p_{Es, en, muc, kr, Gs < 0. ? Es / 4. : Gs} {}
  std::string name() const override { return "HertzContactForceModel"; }
  int law() const override { return GRAINS_GPU_HERTZ; }
  std::vector<double> parameters() const override { return std::vector<double>(p_, p_ + 5); }

 private:
  double p_[5];
};

// HertzMemoryContactForceModel (HertzMemoryContactForceModel.cpp:12-32, 261-309)
class HertzMemoryContactForceModel : public ContactForceModel {
 public:
  HertzMemoryContactForceModel(double Es, double en, double muc, double Gs = -1., double mur = 0.,
                               double etarpf = 0., double epst = 0.)
      : p_{Es, en, muc, Gs < 0. ? Es / 4. : Gs, mur, etarpf, epst} {}
  std::string name() const override { return "HertzMemoryContactForceModel"; }
  int law() const override { return GRAINS_GPU_HERTZ_MEMORY; }
  std::vector<double> parameters() const override { return std::vector<double>(p_, p_ + 7); }

 private:
  double p_[7];
};

// ---- the host image of the particles (AllComponents' active particles) -------
struct ParticleSet {
  std::vector<int32_t> id, shape, material;
  std::vector<double> radius, crust, mass, inertia, position, quaternion, basis, velocity, omega;
  std::vector<double> force, torque;
  std::vector<int32_t> coordination;
  size_t size() const { return id.size(); }
  // adds a particle of shape `shape_id` (from LinkedCellGPU::addShape) and density rho
  void add(int32_t pid, int32_t shape_id, const Convex& cv, double rho, int32_t mat, double crust_thickness,
           const double x[3], const double v[3] = nullptr, const double w[3] = nullptr) {
    id.push_back(pid);
    shape.push_back(shape_id);
    material.push_back(mat);
    double I[6], I1[6];
    cv.BuildInertia(I, I1);
    radius.push_back(cv.computeCircumscribedRadius());
    crust.push_back(crust_thickness);
    mass.push_back(rho * cv.getVolume());  // Particle.cpp:158
    for (int k : {0, 3, 5}) inertia.push_back(I[k] * rho);
    for (int k = 0; k < 3; ++k) {
      position.push_back(x[k]);
      velocity.push_back(v ? v[k] : 0.);
      omega.push_back(w ? w[k] : 0.);
    }
    quaternion.insert(quaternion.end(), {0., 0., 0., 1.});
  }
  grains_gpu_particles view() {
    grains_gpu_particles p{};
    p.n = (int64_t)size();
    p.id = id.data();
    p.shape = shape.data();
    p.material = material.data();
    p.radius = radius.data();
    p.crust = crust.data();
    p.mass = mass.data();
    p.inertia = inertia.data();
    p.position = position.data();
    p.quaternion = quaternion.data();
    p.basis = basis.empty() ? nullptr : basis.data();
    p.velocity = velocity.data();
    p.omega = omega.data();
    return p;
  }
};

// ---- App / AppCollision ------------------------------------------------------
class App {
 public:
  virtual ~App() = default;
  // App::ComputeForces(double time, double dt, list<Particle*> const*) (App.hh:38-39)
  virtual void ComputeForces(double time, double dt, ParticleSet* particles) = 0;
};

class AppCollision : public App {
 public:
  virtual void Link(ParticleSet* particles) = 0;                           // AppCollision::Link(Particle*)
  virtual void LinkUpdate(double time, double dt, ParticleSet* particles) = 0;  // AppCollision::LinkUpdate
};

// LinkedCell on the GPU: broadphase, narrowphase, contact laws and the
// leapfrog integrator of one system (or of an ensemble of independent
// systems) on one device.
class LinkedCellGPU : public AppCollision {
 public:
  explicit LinkedCellGPU(int64_t max_particles, int precision = GRAINS_GPU_MIXED, int device = 0,
                         int n_systems = 1) {
    grains_gpu_config cfg{};
    cfg.precision = precision;
    cfg.device = device;
    cfg.n_systems = n_systems;
    cfg.max_particles = max_particles;
    grains_gpu_ctx* c = nullptr;
    int rc = grains_gpu_create(&cfg, &c);
    ctx_.reset(c);
    check(rc, c);
  }
  grains_gpu_ctx* context() const { return ctx_.get(); }

  // LinkedCell::set (LinkedCell.cpp:47-140); cell_size = 2 * CellSizeFactor * max circumscribed radius
  void set(const double origin[3], const double size[3], double cell_size, const double gravity[3],
           int system = 0) {
    grains_gpu_domain d{};
    for (int k = 0; k < 3; ++k) {
      d.origin[k] = origin[k];
      d.size[k] = size[k];
      d.gravity[k] = gravity[k];
    }
    d.cell_size = cell_size;
    check(grains_gpu_set_domain(ctx_.get(), system, &d), ctx_.get());
  }
  int addShape(const Convex& cv) {
    std::vector<double> p = cv.params();
    int32_t id = -1;
    check(grains_gpu_add_shape(ctx_.get(), cv.getConvexType(), p.data(), (int32_t)p.size(), &id), ctx_.get());
    return id;
  }
  // ContactBuilderFactory::define for the material pair (matA, matB)
  void setContactForceModel(int matA, int matB, const ContactForceModel& m, int system = 0) {
    std::vector<double> p = m.parameters();
    check(grains_gpu_set_contact_law(ctx_.get(), system, matA, matB, m.law(), p.data(), (int32_t)p.size()),
          ctx_.get());
  }
  // AppCollision::Link(Obstacle*) for the obstacles of a system
  void LinkObstacles(const std::vector<grains_gpu_obstacle>& obs, int system = 0) {
    check(grains_gpu_set_obstacles(ctx_.get(), system, (int32_t)obs.size(), obs.data()), ctx_.get());
  }
  // <CollisionDetection Type="GJK" | "GJK_SV">
  void setCollisionAlgorithm(int algorithm) {
    check(grains_gpu_set_collision_algorithm(ctx_.get(), algorithm), ctx_.get());
  }
  // the <ObstacleLoadings> of the input file (ObstacleImposedVelocity)
  void setObstacleLoadings(const std::vector<grains_gpu_obstacle_loading>& loads, int system = 0) {
    check(grains_gpu_set_obstacle_loadings(ctx_.get(), system, (int32_t)loads.size(), loads.data()), ctx_.get());
  }
  void Link(ParticleSet* particles) override {
    grains_gpu_particles v = particles->view();
    check(grains_gpu_upload_particles(ctx_.get(), &v), ctx_.get());
  }
  void LinkUpdate(double time, double dt, ParticleSet*) override {
    check(grains_gpu_link_update(ctx_.get(), time, dt), ctx_.get());
  }
  void ComputeForces(double time, double dt, ParticleSet*) override {
    check(grains_gpu_compute_forces(ctx_.get(), time, dt), ctx_.get());
  }
  // SecondOrderLeapFrog::Move / advanceVelocity over all particles
  void Move(double time, double dt_vel, double dt_disp) {
    check(grains_gpu_move(ctx_.get(), time, dt_vel, dt_disp), ctx_.get());
  }
  void advanceVelocity(double time, double dt_vel) {
    check(grains_gpu_advance_velocity(ctx_.get(), time, dt_vel), ctx_.get());
  }
  // Grains::Simulation's KDK loop for n steps (Grains.cpp:344-364), device resident
  double Simulation(int n_steps, double time, double dt) {
    check(grains_gpu_step(ctx_.get(), n_steps, &time, dt), ctx_.get());
    check(grains_gpu_synchronize(ctx_.get()), ctx_.get());
    return time;
  }
  void initializeLeapFrog(double time, double dt) {
    check(grains_gpu_initialize_leapfrog(ctx_.get(), time, dt), ctx_.get());
  }
  // device -> host image (positions, velocities, forces, coordination...)
  void download(ParticleSet* p) {
    size_t n = p->size();
    p->force.resize(3 * n);
    p->torque.resize(3 * n);
    p->coordination.resize(n);
    p->basis.resize(9 * n);
    grains_gpu_particles v = p->view();
    v.force = p->force.data();
    v.torque = p->torque.data();
    v.coordination = p->coordination.data();
    v.basis = p->basis.data();
    check(grains_gpu_download_particles(ctx_.get(), &v), ctx_.get());
  }
  // the particle file of Grains::saveReload (AllComponents::write, text or hybrid)
  int64_t saveReloadParticles(const std::string& path, bool hybrid = false) {
    int64_t bytes = 0;
    check(grains_gpu_write_reload_particles(ctx_.get(), path.c_str(), hybrid ? 1 : 0, &bytes), ctx_.get());
    return bytes;
  }
  // RawDataPostProcessingWriter::PostProcessing_start (start = true) / PostProcessing
  int64_t writeRawData(const std::string& root, double time, int n_total, bool binary, bool start,
                       int system = 0) {
    int64_t bytes = 0;
    check(grains_gpu_write_rawdata(ctx_.get(), root.c_str(), time, system, n_total, binary ? 1 : 0, start ? 1 : 0,
                                   &bytes),
          ctx_.get());
    return bytes;
  }

 private:
  struct Del {
    void operator()(grains_gpu_ctx* c) const { grains_gpu_destroy(c); }
  };
  std::unique_ptr<grains_gpu_ctx, Del> ctx_;
};

}  // namespace grains_gpu

#endif  // GRAINS_GPU_HPP
