/*
 * grains_gpu.h -- C ABI of the B200 implementation of the Grains3D DEM time
 * step (LinkedCell broadphase, sphere / box / cylinder / polyhedron
 * narrowphase, Hooke and HookeMemory contact laws, second-order leapfrog with
 * quaternion rotation update).
 *
 * Conventions
 *   - Every entry point returns an int status: 0 (GRAINS_GPU_OK) or a bit set
 *     of GRAINS_GPU_* error codes.  The message of the last failure is returned
 *     by grains_gpu_last_error().  The reference signals the same conditions
 *     with C++ exceptions (ContactError, MotionError, SimulationError,
 *     Grains/Base/include/Error.hh:19,75,129); the C++ adaptor in
 *     grains_gpu.hpp rethrows them.
 *   - Plain pointers and sizes only.  All arrays are HOST arrays unless a
 *     function name ends in _device.  Vectors are packed xyz, quaternions
 *     xyzw (vector part first, like Quaternion(x,y,z,w) in
 *     Grains/Geometry/src/Quaternion.cpp:46), 3x3 matrices row major.
 *   - One context per host thread; all work of a context is ordered on its
 *     own CUDA stream.  There is no global mutable state.
 *   - Particle arrays are indexed in upload order.  The device keeps the
 *     particles sorted by cell internally; downloads return upload order.
 */
#ifndef GRAINS_GPU_H
#define GRAINS_GPU_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status bits (reference: Error.hh exceptions + device conditions) --- */
#define GRAINS_GPU_OK                 0
#define GRAINS_GPU_CONTACT_ERROR      (1 << 0) /* ContactError: overlap >= crust sum, RigidBodyWithCrust.cpp:620-629 */
#define GRAINS_GPU_MOTION_ERROR       (1 << 1) /* MotionError: |dx| > crust, Particle.cpp:447-457 */
#define GRAINS_GPU_OUT_OF_GRID        (1 << 2) /* SimulationError: particle left the grid, LinkedCell.cpp:1525-1531 */
#define GRAINS_GPU_PAIR_OVERFLOW      (1 << 3) /* a diagnostic pair buffer was too small */
#define GRAINS_GPU_HISTORY_FULL       (1 << 4) /* more contacts than history slots for one particle */
#define GRAINS_GPU_CUDA_ERROR         (1 << 5)
#define GRAINS_GPU_TIMEOUT            (1 << 6) /* a bounded device wait gave up */
#define GRAINS_GPU_INVALID_ARGUMENT   (1 << 7)
#define GRAINS_GPU_NOT_READY          (1 << 8) /* call order violated (e.g. step before upload) */
#define GRAINS_GPU_GJK_NOT_CONVERGED  (1 << 9) /* GJK hit its iteration cap (Convex.cpp:566) */
#define GRAINS_GPU_CONTACT_HANDLED    (1 << 10) /* informational: a contact went through the crust x10 retry */
#define GRAINS_GPU_CELL_TOO_SMALL     (1 << 11) /* a sphere's diameter exceeds the cell edge: contacts may be missed */

/* ---- enumerations ------------------------------------------------------- */
enum grains_gpu_precision {
  GRAINS_GPU_FP64  = 0, /* everything in double */
  GRAINS_GPU_MIXED = 1  /* positions, quaternions, bases and overlap distances in
                           double; velocities, forces, contact law, history in float */
};

enum grains_gpu_shape_type {   /* Grains/Geometry/include/Convex.hh ConvexType */
  GRAINS_GPU_SPHERE     = 0,   /* params: radius */
  GRAINS_GPU_BOX        = 1,   /* params: LX, LY, LZ (full edge lengths) */
  GRAINS_GPU_CYLINDER   = 2,   /* params: radius, height (axis = local Y) */
  GRAINS_GPU_POLYHEDRON = 3    /* params: nv, nv*(x,y,z), nf, then per face:
                                  k, k vertex indices (reference file format,
                                  Grains/Geometry/src/Polyhedron.cpp:75-115) */
};

enum grains_gpu_contact_law {
  GRAINS_GPU_HOOKE        = 0, /* params: kn, en, etat, muc, kr            (HookeContactForceModel.cpp:170-199) */
  GRAINS_GPU_HOOKE_MEMORY = 1, /* params: kn, en, etat, muc, kt, mur, etarpf, epst
                                                                     (HookeMemoryContactForceModel.cpp:11-29) */
  GRAINS_GPU_HERTZ        = 2, /* params: Es, en, muc, kr, Gs            (HertzContactForceModel.cpp:12-21, 236-276) */
  GRAINS_GPU_HERTZ_MEMORY = 3  /* params: Es, en, muc, Gs, mur, etarpf, epst
                                                               (HertzMemoryContactForceModel.cpp:12-32, 261-309) */
};

/* ---- configuration ------------------------------------------------------ */
typedef struct grains_gpu_config {
  int32_t precision;          /* enum grains_gpu_precision */
  int32_t device;             /* CUDA device ordinal */
  int32_t n_systems;          /* independent systems in one context (>=1) */
  int32_t history_capacity;   /* contact-memory slots per particle, 0 = 24 */
  int64_t max_particles;      /* capacity summed over systems */
  int32_t max_obstacles;      /* capacity summed over systems, 0 = 256 */
  int32_t max_shapes;         /* shape-table capacity, 0 = 64 */
  int32_t max_materials;      /* materials per system, 0 = 4 */
  int32_t reserved[7];
} grains_gpu_config;

/* Domain of one system.  cell_size is the requested linked-cell edge
 * (2 * CellSizeFactor * max circumscribed radius, Grains.cpp:1005-1022,
 * 2522-2526); the grid is built like LinkedCell::set (LinkedCell.cpp:47-140):
 * n_i = int((L_i + 1e-10) / cell_size), edge_i = L_i / n_i.  Periodicity is
 * not supported (out of scope). */
typedef struct grains_gpu_domain {
  double origin[3];
  double size[3];
  double cell_size;
  double gravity[3];
} grains_gpu_domain;

/* Obstacle of one system (a Grains SimpleObstacle).  Obstacles are rigid
 * bodies of mass 1e20 (Component.cpp:16) that are moved by imposed kinematics
 * only.  'moving' != 0 marks an obstacle with imposed motion
 * (ObstacleImposedVelocity.cpp:60-85, 195-208): a ConstantRotation about
 * 'rotation_center' with angular velocity 'omega' when omega is not zero (its
 * centre velocity becomes omega x (centre - rotation_center) at each move),
 * otherwise a ConstantTranslation at 'velocity'. */
typedef struct grains_gpu_obstacle {
  int32_t id;            /* component id (reference obstacles carry their own ids) */
  int32_t shape;         /* shape id from grains_gpu_add_shape (a BOX for walls) */
  int32_t material;
  int32_t moving;
  double  crust;
  double  transform[12]; /* basis (row-major 3x3) then origin, Transform(double m[12]) layout */
  double  velocity[3];
  double  omega[3];
  double  rotation_center[3];
} grains_gpu_obstacle;

/* Imposed obstacle motions (ObstacleImposedVelocity, Component/src/
 * ObstacleImposedVelocity.cpp:60-262 for the XML, 306-455 for the motion):
 * each is active on [t_start, t_end]; over a step ending at time T the active
 * part of [T - dt, T] is integrated analytically, the velocities are those at
 * T, and the motions of all loadings of an obstacle add up
 * (ObstacleKinematicsVelocity::ImposedMotion, ObstacleKinematicsVelocity.cpp:
 * 86-122), in the order of their start times. */
enum grains_gpu_motion {
  GRAINS_GPU_CONSTANT_TRANSLATION = 0,  /* vector = velocity */
  GRAINS_GPU_SIN_TRANSLATION      = 1,  /* vector = direction; amplitude[0] (velocity), period[0], phase_deg[0] */
  GRAINS_GPU_CRENEL_TRANSLATION   = 2,  /* vector = direction; amplitude[0] (velocity), period[0] (half cycle) */
  GRAINS_GPU_CONSTANT_ROTATION    = 3,  /* vector = angular velocity; about center when has_center, else
                                           about the obstacle's own centre */
  GRAINS_GPU_MULTISIN_TRANSLATION = 4,  /* vector = direction; per axis amplitude, period, phase_deg */
  /* An imposed force (ObstacleImposedForce "ConstantTranslation", Component/
   * src/ObstacleImposedForce.cpp:29-80 for the XML, 183-252 for the motion):
   * vector = the force (AX, AY, AZ), amplitude[0] = the virtual mass (<= 0:
   * automatic, dt^2 |F| 1e7 / (2 crust)), amplitude[1] = Vmax.  Each move, a
   * PID controller turns the difference between the contact force on the
   * obstacle (from the last force evaluation) and the imposed force, along
   * the force's direction, into the obstacle's translation over the step; until
   * the contact force first exceeds EPSILON the obstacle moves at -Vmax along
   * the direction.  As in the reference the controller's history is one per
   * system, shared by its force loadings (the reference keeps it in static
   * variables), and the force loadings of an obstacle act in the order given.
   * The reference's "MultiSinTranslation" force has no motion (its body is a
   * "TO DO") and is not offered. */
  GRAINS_GPU_FORCE_TRANSLATION    = 5
};
typedef struct grains_gpu_obstacle_loading {
  int32_t obstacle_id;
  int32_t type;          /* grains_gpu_motion */
  double  t_start, t_end;
  double  vector[3];
  double  center[3];
  int32_t has_center;
  int32_t reserved;
  double  amplitude[3];
  double  period[3];
  double  phase_deg[3];
} grains_gpu_obstacle_loading;

/* Particle state, structure of arrays, n entries each.  Static fields are
 * read by upload only; dynamic fields are read by upload and written by
 * download.  'basis' may be NULL on upload (then basis = R(q)). */
typedef struct grains_gpu_particles {
  int64_t  n;
  int32_t* id;           /* component id, unique within a system, >= 0 */
  int32_t* system;       /* system index, may be NULL when n_systems == 1 */
  int32_t* shape;        /* shape id */
  int32_t* material;
  double*  radius;       /* circumscribed radius (sphere: its radius) */
  double*  crust;        /* crust thickness */
  double*  mass;         /* density * volume, Particle.cpp:158 */
  double*  inertia;      /* 3n: body-frame principal inertia (density scaled), Particle.cpp:159-163 */
  double*  position;     /* 3n: transform origin */
  double*  quaternion;   /* 4n: xyzw */
  double*  basis;        /* 9n: row-major rotation part of the transform (may be NULL) */
  double*  velocity;     /* 3n */
  double*  omega;        /* 3n: world-frame angular velocity */
  double*  force;        /* 3n: download only, current torsor force */
  double*  torque;       /* 3n: download only, current torsor torque */
  int32_t* coordination; /* download only, number of contacting components (Particle.cpp:1703-1707) */
} grains_gpu_particles;

/* Contact memory entries (HookeMemory), reference map
 * Component::m_contactMap (Component.hh:507-513): entry held by component
 * 'owner' about neighbour 'other' (ids; obstacle ids as given). */
typedef struct grains_gpu_contact_memory {
  int64_t  n;
  int32_t* owner;
  int32_t* other;
  double*  kdelta;       /* 3n */
  double*  prev_normal;  /* 3n */
  double*  spring_torque;/* 3n */
  int32_t* system;       /* n: the system of each entry (ids are per system); may be
                            NULL: the download then omits it and an upload puts each
                            entry in the first system that has its owner id */
} grains_gpu_contact_memory;

/* Counters and overlap statistics accumulate over the force evaluations since
 * the last grains_gpu_reset_stats (or the context's creation). */
typedef struct grains_gpu_stats {
  int64_t n_particles;
  int64_t n_candidate_pairs;      /* particle-particle candidates (27-cell neighbourhoods) */
  int64_t n_obstacle_candidates;  /* particle-obstacle candidates after the InZone prefilter */
  int64_t n_contacts;             /* particle-particle contacts */
  int64_t n_obstacle_contacts;
  int64_t n_gjk_calls;
  int64_t n_gjk_iterations;
  double  overlap_max;            /* AppCollision::addToContactsFeatures, AppCollision.cpp:160-187 */
  double  overlap_sum;
  int64_t n_steps_done;
  int32_t status;                 /* accumulated status bits */
  int32_t reserved;
  /* running means since the last reset, as AppCollision::getOverlapMean /
   * getNbIterGJKMean report them (AppCollision.cpp:160-187): the overlap of
   * every contact met, the GJK iterations of every GJK call */
  double  overlap_mean;
  double  gjk_iterations_mean;
} grains_gpu_stats;

typedef struct grains_gpu_ctx grains_gpu_ctx;

/* ---- lifetime ----------------------------------------------------------- */
/* replaces: Grains::Construction creating `new LinkedCell` (Grains.cpp:778-780) */
int grains_gpu_create(const grains_gpu_config* cfg, grains_gpu_ctx** out);
int grains_gpu_destroy(grains_gpu_ctx* ctx);
/* copies the message of the last failure (NUL terminated) */
int grains_gpu_last_error(const grains_gpu_ctx* ctx, char* buf, size_t len);
/* CUDA stream of the context, as a void* (cudaStream_t) */
int grains_gpu_get_stream(const grains_gpu_ctx* ctx, void** stream);

/* ---- set-up ------------------------------------------------------------- */
/* replaces: LinkedCell::set (LinkedCell.cpp:47-140) and the gravity of
 * GrainsExec::m_vgravity */
int grains_gpu_set_domain(grains_gpu_ctx* ctx, int32_t system, const grains_gpu_domain* dom);
/* replaces: ConvexBuilderFactory::create (Grains/Geometry/src/ConvexBuilderFactory.cpp) */
int grains_gpu_add_shape(grains_gpu_ctx* ctx, int32_t type, const double* params,
                         int32_t n_params, int32_t* shape_id);
/* replaces: ContactBuilderFactory::define / defineParameters
 * (ContactBuilderFactory.cpp:81-169); symmetric in (matA, matB) */
int grains_gpu_set_contact_law(grains_gpu_ctx* ctx, int32_t system, int32_t mat_a,
                               int32_t mat_b, int32_t law, const double* params,
                               int32_t n_params);
/* replaces: AppCollision::Link(Obstacle*) / LinkedCell::Link(Obstacle*)
 * (LinkedCell.cpp:1371-1445) */
int grains_gpu_set_obstacles(grains_gpu_ctx* ctx, int32_t system, int32_t n,
                             const grains_gpu_obstacle* obstacles);
/* replaces: ObstacleImposedVelocity loadings of Grains::Construction
 * (<ObstacleLoadings>, ObstacleImposedVelocity.cpp:60-262).  Sets every loading
 * of the system's obstacles (after grains_gpu_set_obstacles); an obstacle with
 * loadings moves by them, one without by its 'moving' / velocity / omega
 * fields (as a single loading from 0 on). */
int grains_gpu_set_obstacle_loadings(grains_gpu_ctx* ctx, int32_t system, int32_t n,
                                     const grains_gpu_obstacle_loading* loadings);
/* replaces: <CollisionDetectionAlgorithm><CollisionDetection Type="GJK" | "GJK_SV">
 * (Base/src/Grains.cpp:640-670, GrainsExec::m_colDetGJK_SV): the distance
 * algorithm of RigidBodyWithCrust::ClosestPoint (RigidBodyWithCrust.cpp:299-312)
 * for pairs of non-spherical bodies, Johnson's (Convex.cpp:536-627, the
 * default) or the signed-volume one (GJK_SV.cpp:428-525).  The crust-x10 retry
 * and the obstacle-cell links use Johnson's, as in the reference. */
enum grains_gpu_collision_algorithm { GRAINS_GPU_GJK = 0, GRAINS_GPU_GJK_SV = 1 };
int grains_gpu_set_collision_algorithm(grains_gpu_ctx* ctx, int32_t algorithm);
/* replaces: the Tolerance, Acceleration and History attributes of
 * <CollisionDetection> (Base/src/Grains.cpp:674-723; GrainsExec::m_colDetTolerance,
 * m_colDetAcceleration, m_colDetWithHistory).
 *   tolerance     relative optimality gap of the GJK runs (>= 1e-10; the
 *                 reference's default is 1e-10)
 *   acceleration  1: Nesterov-accelerated search directions (Convex.cpp:566-597)
 *   history       1: each convex particle pair keeps its last GJK iterate and
 *                 starts its next run from it (CollisionHistory, Particle.cpp:
 *                 486-505; Convex.cpp:636-716).  The history of a pair lives in
 *                 the row of its lower id, one slot per owned work item, up to
 *                 history_capacity of them; a pair beyond that starts cold.
 * Applies to both GJK algorithms and to the crust-x10 retry; the static
 * obstacle-cell links use the tolerance and acceleration too, so set the
 * options before grains_gpu_upload_particles.  Default: 1e-10, 0, 0. */
int grains_gpu_set_collision_options(grains_gpu_ctx* ctx, double tolerance, int32_t acceleration,
                                     int32_t history);
/* replaces: LinkedCell::Link(Particle*) for all active particles
 * (LinkedCell.cpp:1330-1365) + AllComponents state upload */
int grains_gpu_upload_particles(grains_gpu_ctx* ctx, const grains_gpu_particles* p);
int grains_gpu_download_particles(grains_gpu_ctx* ctx, grains_gpu_particles* p);
/* Overwrites the kinematic state (position, quaternion, basis when given,
 * velocity, omega) of the particles already uploaded, in upload order (p->n
 * must equal the uploaded count; static fields are ignored).  Contact memory,
 * forces and set-up tables are kept: this is the per-step host->device path
 * of an adaptor whose host copy of the state stays authoritative, like
 * AllComponents in the reference (AllComponents.cpp:151-233). */
int grains_gpu_update_particles(grains_gpu_ctx* ctx, const grains_gpu_particles* p);
/* The kinematic state of some of the uploaded particles: rows[k] (distinct
 * upload indices) gets entry k of p's position, quaternion, basis (when given),
 * velocity and omega arrays (n_rows entries each; p->n is ignored); the other
 * particles keep theirs untouched.  The ghost refresh of a domain-decomposed
 * run overwrites only its ghosts this way, as the reference's
 * GrainsMPIWrapper::UpdateClones updates only the clones
 * (GrainsMPIWrapper.cpp:1556-1684). */
int grains_gpu_update_particle_rows(grains_gpu_ctx* ctx, int64_t n_rows, const int64_t* rows,
                                    const grains_gpu_particles* p);
/* replaces: Particle::setFluidDensity / setFluidCorrectedAcceleration with
 * AllComponents::computeWeight and setParticlesCouplingFactor (Particle.cpp:
 * 414-419, 820-825, 1284-1288; ParticleKinematics.cpp:483-488), the fluid
 * set-up of GrainsCoupledWithFluid (Fluid/src/GrainsCoupledWithFluid.cpp:
 * 1200-1207).  Immersed particles: the weight becomes m (1 - rho_f / rho_p) g
 * and, when corrected != 0, the translational and angular accelerations are
 * divided by 1 - rho_f / rho_p (SecondOrderLeapFrog.cpp:50-52,
 * ParticleKinematics3D.cpp:64-69).  particle_density: rho_p in upload order
 * (n values; may be null when fluid_density is 0, which switches the fluid
 * off).  Set after grains_gpu_upload_particles; an upload clears it. */
int grains_gpu_set_fluid(grains_gpu_ctx* ctx, double fluid_density, int32_t corrected,
                         const double* particle_density);
/* replaces: AppPRSHydroFT::setHydroFT + ComputeForces (Fluid/src/
 * AppPRSHydroFT.cpp:29-73): a force (at the centre) and a torque per particle,
 * 3 doubles each in upload order, added to every force evaluation after the
 * contact forces until set again; both null removes them.  An upload clears
 * them. */
int grains_gpu_set_hydro_forces(grains_gpu_ctx* ctx, const double* force, const double* torque);
/* replaces: GrainsCoupledWithFluid::updateParticlesVelocity (Fluid/src/
 * GrainsCoupledWithFluid.cpp:1126-1185): translational and angular velocity
 * (world frame) of every particle, 3 doubles each in upload order. */
int grains_gpu_set_velocities(grains_gpu_ctx* ctx, const double* velocity, const double* omega);
/* replaces: GrainsCoupledWithFluid::Simulation(dt_fluid) (Fluid/src/
 * GrainsCoupledWithFluid.cpp:123-229): the DEM steps of one fluid step.
 * dteff = max(min(max_dt, dt_fluid / *ndt), min_dt); *ndt becomes
 * (size_t)(dt_fluid / dteff) (the count carries over to the next call, as
 * m_ndt does) and *ndt kick-drift-kick steps of dt_fluid / *ndt run
 * (grains_gpu_step); *time advances by dt_fluid. */
int grains_gpu_fluid_step(grains_gpu_ctx* ctx, double dt_fluid, double min_dt, double max_dt, int64_t* ndt,
                          double* time);
/* replaces: GrainsCoupledWithFluid::GrainsToFluid (Fluid/src/
 * GrainsCoupledWithFluid.cpp:912-1120) as GrainsToBasilisk passes it on
 * (InterfaceCBasilisk/src/InterfaceGrains3DBasilisk.cpp:64-87): the rigid
 * bodies for the fluid solver as one line of space-separated tokens (each
 * followed by one space).  Per particle, by increasing id: index, corner code
 * (Convex::getNbCorners: 1 sphere, 666 box, 777 cylinder, vertex count
 * polyhedron), "P", velocity, angular velocity, density, mass, the
 * space-fixed inertia tensor (xx xy xz yy yz zz), the rotation matrix, the
 * centre, the circumscribed radius, then the envelope points in world
 * coordinates and the faces (RigidBody::writePositionInFluid).  *len = the
 * size with the terminating 0; buf may be null to query it. */
int grains_gpu_fluid_features(grains_gpu_ctx* ctx, char* buf, int64_t cap, int64_t* len);
/* No counterpart in the reference: attaches a context set up through this
 * interface to the fluid solvers' C interface below, with the time-step
 * bounds of <Simulation><TimeStep mindt maxdt ndt> (GrainsCoupledWithFluid.cpp:
 * 509-531).  The reference builds its coupled simulation from its XML and
 * reload files in Init_Grains; that input layer is the host's here. */
int grains_gpu_basilisk_attach(grains_gpu_ctx* ctx, double min_dt, double max_dt, int64_t ndt);
/* The fluid solvers' C interface, same names and signatures as
 * InterfaceCBasilisk/include/InterfaceGrains3DBasilisk.h:12-30, driving the
 * attached context.  Init_Grains applies the fluid density and the
 * acceleration correction (its input file name and restart flag are not
 * read) and starts the leapfrog; Simu_Grains = grains_gpu_fluid_step;
 * GrainsToBasilisk = grains_gpu_fluid_features in a malloc'ed string (free
 * it); UpdateVelocityGrains sets the velocities from an m x 6 array ordered by
 * id; NumberOfRigidBodiesInBasilisk reports the particles and no obstacle.
 * SaveResults_Grains and checkParaviewPostProcessing_Grains write nothing
 * (the Paraview writers are out of scope).  Like the reference, errors end
 * the process with a message. */
void Init_Grains(char const* inputfile, double fluid_rho, const bool b_restart, const bool b_fluidcorrectedacc);
void Simu_Grains(const double dt_fluid);
char* GrainsToBasilisk(int* pstrsize);
void SetInitialTime(double tinit);
void SaveResults_Grains(void);
void checkParaviewPostProcessing_Grains(char* solid_resDir);
void UpdateVelocityGrains(double** arrayv, const int m);
void SetInitialCycleNumber(int cycle0);
void NumberOfRigidBodiesInBasilisk(size_t* nparticles, size_t* nobstacles);
int grains_gpu_upload_contact_memory(grains_gpu_ctx* ctx, const grains_gpu_contact_memory* m);
/* n on input = capacity; on output = number of entries written (owner-side
 * and mirrored entries both listed, like the reference's two maps) */
int grains_gpu_download_contact_memory(grains_gpu_ctx* ctx, grains_gpu_contact_memory* m);
/* obstacle poses after imposed motion: 12 doubles per obstacle of 'system' */
int grains_gpu_download_obstacles(grains_gpu_ctx* ctx, int32_t system, int32_t n,
                                  double* transforms);

/* ---- the time step ------------------------------------------------------ */
/* replaces: App::ComputeForces(time, dt, particles) of LinkedCell
 * (App.hh:38-39, LinkedCell.cpp:1019-1103) together with the per-step resets
 * of Grains::computeParticlesForceAndTorque (Grains.cpp:459-482) */
int grains_gpu_compute_forces(grains_gpu_ctx* ctx, double time, double dt);
/* replaces: AllComponents::Move (AllComponents.cpp:151-222) ->
 * SecondOrderLeapFrog::Move (SecondOrderLeapFrog.cpp:44-69), obstacle motion.
 * time = the clock after this step's increment (Grains::Simulation adds dt to
 * m_time before the move); imposed obstacle motion acts over the interval
 * time - (time - dt_disp), as in ObstacleImposedVelocity::isActif. */
int grains_gpu_move(grains_gpu_ctx* ctx, double time, double dt_vel, double dt_disp);
/* replaces: AppCollision::LinkUpdate (LinkedCell.cpp:1452-1547) */
int grains_gpu_link_update(grains_gpu_ctx* ctx, double time, double dt);
/* replaces: AllComponents::advanceParticlesVelocity ->
 * SecondOrderLeapFrog::advanceVelocity (SecondOrderLeapFrog.cpp:74-95) */
int grains_gpu_advance_velocity(grains_gpu_ctx* ctx, double time, double dt_vel);
/* The leapfrog initialisation of Grains::do_before_time_stepping
 * (Grains.cpp:169-174): one force evaluation, then kdelta and the rolling
 * spring torque of every memory entry are zeroed. */
int grains_gpu_initialize_leapfrog(grains_gpu_ctx* ctx, double time, double dt);
/* n_steps kick-drift-kick steps of Grains::Simulation (Grains.cpp:344-364),
 * replayed from a CUDA graph.  *time is advanced by n_steps*dt. */
int grains_gpu_step(grains_gpu_ctx* ctx, int32_t n_steps, double* time, double dt);
/* blocks until the stream is idle; returns accumulated device status bits */
int grains_gpu_synchronize(grains_gpu_ctx* ctx);

/* ---- diagnostics -------------------------------------------------------- */
/* Candidate pairs of the current cell assignment (LinkedCell::ComputeForces
 * enumeration as a set): pairs[2k], pairs[2k+1] = ids with pairs[2k] <
 * pairs[2k+1], sorted.  Obstacle candidates follow with the obstacle id in
 * the second slot when include_obstacles != 0.  *n = pairs found (may exceed
 * cap, then GRAINS_GPU_PAIR_OVERFLOW). */
int grains_gpu_get_candidate_pairs(grains_gpu_ctx* ctx, int32_t system, int32_t include_obstacles,
                                   int64_t cap, int32_t* pairs, int64_t* n);
/* Contact pairs (overlap distance < 0) of system `system` in the last force
 * evaluation of grains_gpu_compute_forces, same layout (ids are per system). */
int grains_gpu_get_contact_pairs(grains_gpu_ctx* ctx, int32_t system, int64_t cap,
                                 int32_t* pairs, int64_t* n);
/* Contact pairs of system `system` in the last force evaluation of
 * grains_gpu_compute_forces with the contact force (delFN + delFT of the contact law) on the lower id of
 * each: forces[3k..3k+2] for pairs[2k], pairs[2k+1], same order as
 * grains_gpu_get_contact_pairs.  The reference applies the same force at the
 * contact point through Component::addForce (Component.cpp:67-71) inside
 * HookeMemoryContactForceModel::computeForces (:200-249); it keeps no list. */
int grains_gpu_get_contact_forces(grains_gpu_ctx* ctx, int32_t system, int64_t cap, int32_t* pairs,
                                  double* forces, int64_t* n);
int grains_gpu_get_stats(grains_gpu_ctx* ctx, grains_gpu_stats* st);
/* Reset the accumulated status bits and statistics. */
int grains_gpu_reset_stats(grains_gpu_ctx* ctx);

/* ---- tuning ---------------------------------------------------------------- */
/* No counterpart in the reference (its grid is fixed by CellSizeFactor and it
 * has no launch shapes).  Launch and grid choices of a context, none of which
 * changes contacts or forces beyond the order of floating-point sums:
 *   cell_factor    linked-cell edge = cell_factor x the domain's cell_size
 *                  (1 = LinkedCell::set's grid; 1 .. 4).  Candidate pairs
 *                  (a diagnostic) follow the grid.
 *   contacts_block threads per block of the broadphase kernel (32 .. 256)
 *   forces_block   threads per block of the contact-law kernel (32 .. 128)
 *   list_capacity  contact-list slots per particle (8 .. 256, a multiple
 *                  of 4; 0 = 32 for spheres, 64 when other shapes are
 *                  present): contacting particles and candidate obstacles of
 *                  a force evaluation; a particle with more fails the step
 *                  with GRAINS_GPU_PAIR_OVERFLOW
 *   gather_every   steps between two permutations of the particle arrays
 *                  into cell order (1 .. 64); in between the cell lists are
 *                  rebuilt every step and reached through a permutation.
 *                  Results do not depend on it: every sum runs in cell order,
 *                  then id order inside a cell.
 *   persistent     1: the middle steps of grains_gpu_step run in one
 *                  cooperative launch (every block resident, the phases
 *                  separated by a grid barrier with a bounded wait) instead of
 *                  6 launches per step replayed from graphs; same results.
 *                  Pays where launch gaps dominate (small systems). */
typedef struct grains_gpu_tuning {
  double  cell_factor;
  int32_t contacts_block;
  int32_t forces_block;
  int32_t list_capacity;
  int32_t gather_every;
  int32_t persistent;
  int32_t reserved[3];
} grains_gpu_tuning;
int grains_gpu_get_tuning(const grains_gpu_ctx* ctx, grains_gpu_tuning* tuning);
int grains_gpu_set_tuning(grains_gpu_ctx* ctx, const grains_gpu_tuning* tuning);
/* Autotuner: times trial_steps fused steps from the context's current state
 * for candidate tunings (coordinate descent over list capacity, force block,
 * broadphase block, cell factor), keeps the fastest that completed without
 * error, applies it and restores the state exactly (particles, contact
 * memory, obstacle poses).  The candidates cover the list capacity, the two
 * block shapes, the gather period and the cell factor (coordinate descent).
 * time = the current simulation time. */
int grains_gpu_autotune(grains_gpu_ctx* ctx, double time, double dt, int32_t trial_steps,
                        grains_gpu_tuning* best, double* best_ms);

/* ---- timing helpers for benchmarks ---------------------------------------- */
/* Times each phase of n_steps uncaptured steps with CUDA events on the
 * context stream: first_move, sort_gather, contacts, pairs (with the GJK
 * kernel of convex scenarios), sums_kick (the per-particle sums with the
 * second half kick and the next step's first half kick, drift and binning),
 * obstacle_move (the moving obstacles' kernel).
 * names: '\n'-separated phase names (cap bytes); ms[k]: total milliseconds of
 * phase k; launches[k]: its kernel launches. */
int grains_gpu_profile_kernels(grains_gpu_ctx* ctx, int32_t n_steps, double* time, double dt,
                               char* names, size_t cap, double* ms, int64_t* launches,
                               int32_t max_kernels, int32_t* n_kernels);
/* No counterpart in the reference: a test hook of the persistent launch's
 * failure path.  polls = how many times a grid-barrier wait polls before it
 * gives up (default 2^24, about a second), skip_block = a block that leaves the
 * kernel before its first barrier (-1 = none), so that the other blocks' waits
 * run out: they set GRAINS_GPU_TIMEOUT and return, and the context stays
 * usable (upload the state again before stepping on). */
int grains_gpu_set_barrier_test(grains_gpu_ctx* ctx, int64_t polls, int32_t skip_block);
/* Kernel launches of one middle step of grains_gpu_step: the cell sort (3:
 * the tile-local scan, the scatter, the cell sort), contacts, the GJK phase of
 * convex scenarios with Johnson's GJK (two kernels grouping the GJK items by
 * shape pair, the GJK kernel), pairs, the sums with the kick, the contact
 * forces on force-driven obstacles when there are some, and the obstacle
 * move when obstacles move.  The permutation of the arrays into cell order
 * adds one launch every gather_every steps (grains_gpu_tuning). */
int grains_gpu_launches_per_step(grains_gpu_ctx* ctx, int64_t* launches);

/* ---- allocation-free contact detection ------------------------------------- */
/* No counterpart in the reference: an allocation-free variant of the contact
 * detection of grains_gpu_compute_forces for callers that cannot call
 * cudaMalloc (code inside a stream capture that must not allocate, real-time
 * loops that cannot afford cudaMalloc's implicit synchronisation, hosts that
 * own all device memory through their own pool).  It bins n spheres into the
 * linked-cell grid of (origin, size, cell_size) (LinkedCell::set rules), sorts
 * them by cell and writes every pair of input indices (i < j) whose overlap
 * distance |x_j - x_i| - (r_i + r_j) is negative, decided in double precision
 * exactly like the context-based path.
 *   position (3n doubles), radius (n doubles): device arrays, current device
 *   pairs: device, 2*cap int32; *n_pairs (device int64) = pairs found (may
 *     exceed cap: only cap are written); *status (device int32) = status bits
 *     of this call: GRAINS_GPU_OUT_OF_GRID for a sphere outside the grid,
 *     GRAINS_GPU_CELL_TOO_SMALL when a sphere's diameter exceeds the smallest
 *     cell edge (only the 27 surrounding cells are searched, so contacts may
 *     then be missed: pass a cell_size of at least the largest diameter)
 *   stream: cudaStream_t (NULL = legacy default stream); the call is
 *     asynchronous on it.
 * Only the set of pairs is defined: their order in `pairs` comes from device
 * atomics and changes from call to call.
 * Limits: n <= 65,536 spheres and at most 262,144 cells; larger inputs, and
 * non-finite or non-positive sizes, return GRAINS_GPU_INVALID_ARGUMENT without
 * launching anything.  The scratch (4,980,752 bytes, about 5.0 MB) is a
 * file-scope device array present on every GPU that loads the library until
 * the process exits; every call on a device shares it, so calls that overlap
 * on the GPU (different streams, or several host threads) race and must be
 * serialised by the caller.  A call outside a stream capture looks up the
 * array's device address (cudaGetSymbolAddress); a call inside a capture uses
 * the address the last call outside one found, so make a first call on each
 * device before any stream capture (a first call inside one returns
 * GRAINS_GPU_NOT_READY), and again after a cudaDeviceReset.  No cudaMalloc,
 * cudaFree or allocating library routine is called.  Nothing has to start at
 * zero: each call clears *n_pairs, *status and the part of the scratch it uses
 * before it writes them. */
int grains_gpu_sphere_contacts_noalloc(int32_t n, const double* position, const double* radius,
                                       const double origin[3], const double size[3], double cell_size,
                                       int32_t* pairs, int64_t cap, int64_t* n_pairs, int32_t* status,
                                       void* stream);

/* ---- gradients: differentiable run and its adjoint ------------------------ */
/* No counterpart in the reference (Grains3D has no gradients).  A handle on a
 * context whose particles are uploaded: spheres with static box walls, Hooke
 * or HookeMemory laws, one or more systems.
 *
 * grains_gpu_adjoint_forward runs the leapfrog of Grains::Simulation
 * (Grains.cpp:169-174, 344-364) for n_steps from the context's current state,
 * with the context's contact laws: the leapfrog start (one force evaluation,
 * then kdelta and rolling springs of new memory entries zeroed), n_steps
 * kick-drift-kick steps and the final half kick.  The context's own state is
 * not changed.  The contact memory starts empty.  It keeps a checkpoint (state
 * and contact rows) every 'checkpoint_every' force evaluations and a tape of
 * one segment; the final positions, velocities and angular velocities (world
 * frame) are written to the host arrays (3n doubles each, upload order; any
 * may be NULL).  Contact pairs are owned by the lower upload index.
 *
 * grains_gpu_adjoint_backward takes dL/d(final position, velocity, angular
 * velocity) (3n doubles each, upload order, NULL = zero) and returns
 * dL/d(initial position, velocity, angular velocity) and, in grad_laws, 4
 * doubles per law-table slot: dL/d(kn, en, muc, kt).  Slot of the law used by
 * a contact whose owner has material a and partner material b (a wall's
 * material for walls) in system s: (s * M + a) * M + b, M = max_materials of
 * the context; a law set for (a, b) with a != b is used through both (a, b)
 * and (b, a), so its gradient is the sum of the two slots.  Gradients are of
 * the discrete map (exact up to the precision of the context: FP32 adjoint in
 * mixed precision), valid away from contact onset / release events.
 * Errors of the run (ContactError, MotionError, out of grid, more contacts
 * than history_capacity) fail the call. */
typedef struct grains_gpu_adjoint grains_gpu_adjoint;
int grains_gpu_adjoint_create(grains_gpu_ctx* ctx, int32_t checkpoint_every, grains_gpu_adjoint** out);
int grains_gpu_adjoint_destroy(grains_gpu_adjoint* adj);
int grains_gpu_adjoint_last_error(const grains_gpu_adjoint* adj, char* buf, size_t len);
int grains_gpu_adjoint_law_slots(const grains_gpu_adjoint* adj, int32_t* n_slots);
int grains_gpu_adjoint_forward(grains_gpu_adjoint* adj, int32_t n_steps, double dt, double* position,
                               double* velocity, double* omega);
/* Signature of the contact sets of the last forward run: the xor of a 64-bit
 * hash of every (force evaluation, owner, partner, branch of the contact law)
 * contact, and the number of contacts summed over the evaluations.  Two runs
 * with equal signatures met the same contacts at the same steps, each in the
 * same case of the law (tangential direction from the velocity or from the
 * spring; stick or Coulomb slip): the condition under which the run is smooth
 * between them and finite differences approximate its gradient. */
int grains_gpu_adjoint_contact_signature(const grains_gpu_adjoint* adj, uint64_t* signature, int64_t* n_contacts);
int grains_gpu_adjoint_backward(grains_gpu_adjoint* adj, const double* dl_dposition, const double* dl_dvelocity,
                                const double* dl_domega, double* grad_position, double* grad_velocity,
                                double* grad_omega, double* grad_laws, int32_t n_grad_laws);

/* ---- reload and RawData files --------------------------------------------- */
/* Attributes that the reference's reload files carry per particle and the step
 * does not use (Particle::write2014, Particle.cpp:1146-1157), in upload order:
 * m_GeomType (index of the particle's reference type), tag (0 interior,
 * 1 buffer zone, 2 periodic clone), activity (1 = COMPUTE) and the transform
 * type bits of Transform.hh:246-260.  Any array may be NULL (kept).  An upload
 * sets the shape id, 0, 1 and TRANSLATION (1); a move adds ROTATION and
 * TRANSLATION, as Transform::composeLeftByRotation / setOrigin do. */
int grains_gpu_set_record_attributes(grains_gpu_ctx* ctx, int64_t n, const int32_t* geom_type, const int32_t* tag,
                                     const int32_t* active, const int32_t* transform_type);

/* The particle file of a __Format2024__ reload (AllComponents::write,
 * AllComponents.cpp:1148-1180; Grains::saveReload, Base/src/Grains.cpp:2541-2580
 * writes the header file that names it): binary = 0 writes "Text" mode, one
 * Particle::write2014 line per particle (Particle.cpp:1146-1157); binary = 1
 * writes "Hybrid" mode, per particle its byte count (size_t) then
 * Particle::write2014_binary (Particle.cpp:1183-1195).  Particles in upload
 * order; each carries its contact map (Component::writeContactMemory2014,
 * Component.cpp:776-835) with both sides of every pair, as the reference keeps
 * them (Component.cpp:675-684), sorted by neighbour id.  Numbers are formatted
 * on the device exactly as GrainsExec::doubleToString(ios::scientific, 16, x)
 * prints them (Base/src/GrainsExec.cpp:213-225).  *bytes = file size. */
int grains_gpu_write_reload_particles(grains_gpu_ctx* ctx, const char* path, int32_t binary, int64_t* bytes);

/* One output time of RawDataPostProcessingWriter::one_output_Standard
 * (PostProcessing/src/RawDataPostProcessingWriter.cpp:369-600) for one system:
 * appends (truncate = 0) or starts (truncate = 1, the reference's "new" run)
 * <root>_position_{x,y,z}.dat, _translational_velocity_{x,y,z}.dat,
 * _angular_velocity_{x,y,z}.dat, _coordinationNumber.dat, and rewrites
 * <root>_particleType.dat.  Columns are particle ids 1..n_total; absent ids
 * and periodic clones get the reference's inactive values.  Text (6 digits)
 * or binary (WritingMode="Binary"). *bytes = bytes written. */
int grains_gpu_write_rawdata(grains_gpu_ctx* ctx, const char* root, double time, int32_t system, int32_t n_total,
                             int32_t binary, int32_t truncate, int64_t* bytes);

/* A particle file read back (Particle::read2014 / read2014_binary,
 * Particle.cpp:972-1072; AllComponents::read_particles).  The parse is done
 * at grains_gpu_reload_open; grains_gpu_reload_get reports the counts and copies
 * the arrays that are not NULL (capacity n_particles / n_memory entries).
 * Quaternions are xyzw.  Memory entries: every contact-map entry with its
 * holder's id as owner (both sides of each pair, as in the file);
 * grains_gpu_upload_contact_memory keeps the side it needs. */
typedef struct grains_gpu_reload grains_gpu_reload;
typedef struct grains_gpu_reload_data {
  int64_t  n_particles;
  int64_t  n_memory;
  int32_t* geom_type;
  int32_t* id;
  int32_t* tag;
  int32_t* active;
  int32_t* transform_type;
  double*  position;      /* 3n */
  double*  basis;         /* 9n, row-major */
  double*  velocity;      /* 3n */
  double*  quaternion;    /* 4n */
  double*  omega;         /* 3n */
  double*  force;         /* 3n */
  double*  torque;        /* 3n */
  grains_gpu_contact_memory memory;
} grains_gpu_reload_data;
int grains_gpu_reload_open(const char* path, int32_t binary, grains_gpu_reload** out);  /* *out set even on failure */
int grains_gpu_reload_last_error(const grains_gpu_reload* r, char* buf, size_t len);
int grains_gpu_reload_get(const grains_gpu_reload* r, grains_gpu_reload_data* out);
int grains_gpu_reload_close(grains_gpu_reload* r);

/* GrainsExec::doubleToString(ios::scientific, digits, x) (Base/src/GrainsExec.cpp:
 * 213-225) on the host, with the device writers' formatter: writes the text
 * and a NUL into out; *length = its length.  0 <= digits <= 16. */
int grains_gpu_format_double(double x, int32_t digits, char* out, size_t cap, int32_t* length);

/* The same formatter on the device: the n values, each followed by '\n',
 * formatted on the current device; *length = bytes written to out (host). */
int grains_gpu_format_doubles(const double* x, int64_t n, int32_t digits, char* out, int64_t cap,
                              int64_t* length);

/* ---- shape helpers (reference geometry formulas, host only) -------------- */
/* volume, circumscribed radius and body-frame principal inertia per unit
 * density: Sphere.cpp:61-81,152-155; Box.cpp:181-210; Cylinder.cpp:61-85;
 * Polyhedron.cpp:324-367. */
int grains_gpu_shape_properties(int32_t type, const double* params, int32_t n_params,
                                double* volume, double* circumscribed_radius,
                                double inertia[3]);

#ifdef __cplusplus
}
#endif
#endif /* GRAINS_GPU_H */
