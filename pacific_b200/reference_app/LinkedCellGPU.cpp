// LinkedCellGPU.cpp -- the drop-in collision App of Grains3D on B200 (see
// LinkedCellGPU.hh).
#include "LinkedCellGPU.hh"

#include <string>

#include "Error.hh"
#include "Particle.hh"
#include "Quaternion.hh"
#include "grains_gpu.h"

LinkedCellGPU::LinkedCellGPU(grains_gpu_ctx* ctx) : LinkedCell(), m_ctx(ctx) {
  // the device's ids are the reference ids unless setRows says otherwise
  grains_gpu_particles p{};
  std::vector<int32_t> id(1 << 20);
  p.n = (int64_t)id.size();
  p.id = id.data();
  check(grains_gpu_download_particles(m_ctx, &p));
  for (int64_t i = 0; i < p.n; ++i) m_row[id[i]] = (int)i;
}

LinkedCellGPU::~LinkedCellGPU() {}

void LinkedCellGPU::setRows(std::map<int, int> const& row_of_id) { m_row = row_of_id; }

void LinkedCellGPU::check(int rc) const {
  if (rc == GRAINS_GPU_OK) return;
  char buf[512] = {0};
  grains_gpu_last_error(m_ctx, buf, sizeof(buf));
  // the reference's exceptions, as its time loop catches them (Error.hh)
  if (rc & GRAINS_GPU_CONTACT_ERROR) throw ContactError();
  if (rc & GRAINS_GPU_MOTION_ERROR) throw MotionError();
  if (rc & GRAINS_GPU_OUT_OF_GRID) throw SimulationError();
  throw SimulationError();
}

void LinkedCellGPU::ComputeForces(double time, double dt, list<Particle*> const* particles) {
  const size_t n = m_row.size();
  m_position.resize(3 * n);
  m_quaternion.resize(4 * n);
  m_velocity.resize(3 * n);
  m_omega.resize(3 * n);
  m_force.resize(3 * n);
  m_torque.resize(3 * n);
  for (Particle* P : *particles) {
    auto it = m_row.find(P->getID());
    if (it == m_row.end()) continue;
    const size_t i = (size_t)it->second;
    Point3 const* x = P->getPosition();
    Quaternion const* q = P->getQuaternionRotation();
    Vector3 const* v = P->getTranslationalVelocity();
    Vector3 const* w = P->getAngularVelocity();
    for (int k = 0; k < 3; ++k) {
      m_position[3 * i + k] = (*x)[k];
      m_velocity[3 * i + k] = (*v)[k];
      m_omega[3 * i + k] = (*w)[k];
    }
    Vector3 const* qv = q->getVector3();
    m_quaternion[4 * i] = (*qv)[0];
    m_quaternion[4 * i + 1] = (*qv)[1];
    m_quaternion[4 * i + 2] = (*qv)[2];
    m_quaternion[4 * i + 3] = q->getdouble();
  }
  grains_gpu_particles up{};
  up.n = (int64_t)n;
  up.position = m_position.data();
  up.quaternion = m_quaternion.data();
  up.velocity = m_velocity.data();
  up.omega = m_omega.data();
  check(grains_gpu_update_particles(m_ctx, &up));
  // the first evaluation of a run is the leapfrog start: forces, then the
  // springs of the contact memory zeroed (Grains.cpp:169-174)
  check(m_started ? grains_gpu_compute_forces(m_ctx, time, dt) : grains_gpu_initialize_leapfrog(m_ctx, time, dt));
  m_started = true;
  grains_gpu_particles down{};
  down.n = (int64_t)n;
  down.force = m_force.data();
  down.torque = m_torque.data();
  check(grains_gpu_download_particles(m_ctx, &down));
  // the torsor holds the weight (InitializeForces, Particle.cpp:1409-1416):
  // add what the device found on top of it
  for (Particle* P : *particles) {
    auto it = m_row.find(P->getID());
    if (it == m_row.end()) continue;
    const size_t i = (size_t)it->second;
    Vector3 const* f0 = P->getForce();
    Vector3 const* t0 = P->getTorque();
    P->addBodyForce(Vector3(m_force[3 * i] - (*f0)[0], m_force[3 * i + 1] - (*f0)[1], m_force[3 * i + 2] - (*f0)[2]));
    P->addTorque(Vector3(m_torque[3 * i] - (*t0)[0], m_torque[3 * i + 1] - (*t0)[1], m_torque[3 * i + 2] - (*t0)[2]),
                 0);
  }
}

void LinkedCellGPU::LinkUpdate(double time, double dt, list<Particle*>* particles) {
  // LinkedCell::LinkUpdate (LinkedCell.cpp:1452-1547): particles no longer
  // active leave the list of active particles
  for (list<Particle*>::iterator p = particles->begin(); p != particles->end();) {
    if ((*p)->getActivity() == COMPUTE) ++p;
    else p = particles->erase(p);
  }
}
