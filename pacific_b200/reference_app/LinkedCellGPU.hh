// LinkedCellGPU.hh -- the drop-in collision App of Grains3D on B200.
//
// Compiled against the reference's own headers (Base/include/LinkedCell.hh,
// AppCollision.hh:79-100, App.hh:38-39) and registered where Grains creates its
// LinkedCell (Base/src/Grains.cpp:777-780): the first App of Grains::m_allApp,
// called each step by Grains::computeParticlesForceAndTorque (Grains.cpp:474-476)
// with the active particles, and by Grains::moveParticlesAndObstacles for the
// relink (Grains.cpp:516).  The time loop, the particles (list<Particle*>) and
// their integration stay the reference's; the broadphase, narrowphase and
// contact law run on the GPU through the C ABI of grains_gpu.h.
//
// Each ComputeForces pushes the particles' kinematic state to the device
// (grains_gpu_update_particles), evaluates the contact forces there
// (grains_gpu_compute_forces: the contact memory stays on the device, like
// each Component's contact map in the reference) and adds the contact force
// and torque of every particle to its torsor, on top of the weight that
// Grains::computeParticlesForceAndTorque put there (InitializeForces).  Device
// errors are rethrown as the reference's ContactError, MotionError or
// SimulationError, which the time loop catches (Grains.cpp:423-450).
// LinkUpdate keeps the reference's bookkeeping of inactive particles; the
// device bins the particles itself, so the host cell lists are not rebuilt.
//
// The device context is set up by the host with the same shapes, contact laws
// and obstacles (static walls: the device context holds its own obstacle
// poses) and the particles in some upload order; setRows tells which upload
// row holds the particle of each reference id (by default the device ids are
// the reference ids).
#ifndef _LINKEDCELLGPU_HH_
#define _LINKEDCELLGPU_HH_

#include <map>
#include <vector>

#include "LinkedCell.hh"

struct grains_gpu_ctx;

class LinkedCellGPU : public LinkedCell {
 public:
  /** @brief The App over a device context that holds the particles */
  explicit LinkedCellGPU(grains_gpu_ctx* ctx);
  ~LinkedCellGPU();

  /** @brief Upload row of the particle of each reference id */
  void setRows(std::map<int, int> const& row_of_id);

  /** @brief The next force evaluation starts a leapfrog run: after it the
      cumulative features of the contact memory (tangential and rolling
      springs) are zeroed, as Grains does with
      AllComponents::setAllContactMapCumulativeFeaturesToZero after the first
      force evaluation of a run (Grains.cpp:169-174).  The first evaluation of
      an App always does. */
  void restartLeapfrog() { m_started = false; }

  /** @brief App::ComputeForces: contact forces and torques of the active
      particles, added to their torsors */
  void ComputeForces(double time, double dt, list<Particle*> const* particles);

  /** @brief AppCollision::LinkUpdate: inactive particles leave the list; the
      device bins the others at the next force evaluation */
  void LinkUpdate(double time, double dt, list<Particle*>* particles);

 private:
  void check(int rc) const;
  grains_gpu_ctx* m_ctx;
  bool m_started = false;    // a force evaluation of this run has been done
  std::map<int, int> m_row;  // reference id -> upload row
  std::vector<double> m_position, m_quaternion, m_velocity, m_omega, m_force, m_torque;
};

#endif
