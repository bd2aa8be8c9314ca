// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.  Exposes the reference Grains3D
// (compiled from its own sources by oracle/ref/Makefile) through the C
// contract of include/grains_gpu.h with the prefix grains_ref_, so that the
// tests and the CPU-baseline leg of bench.py can drive the real reference
// exactly like the CUDA library and the oracle restatement.
//
// A context writes a reference input file (Grains3D XML: LinkedCell, contact
// force models, one particle class per distinct sphere/shape, box obstacles,
// gravity) and a particle-position file, builds the simulation with
// Grains::do_before_time_stepping (Base/src/Grains.cpp:95-179, insertion at
// the initial time from the file), then overwrites the kinematic state and
// the contact memory with the uploaded values through the reference's own
// setters.  Steps go through the reference's Grains::moveParticlesAndObstacles,
// computeParticlesForceAndTorque and AllComponents::advanceParticlesVelocity.
//
// The reference keeps process-wide static state (factories, counters), so one
// context per process is supported.
#include "../../include/grains_gpu.h"
#include "LinkedCellGPU.hh"

#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "AllComponents.hh"
#include "Cell.hh"
#include "Component.hh"
#include "ContactBuilderFactory.hh"
#include "Grains.hh"
#include "GrainsBuilderFactory.hh"
#include "GrainsExec.hh"
#include "LinkedCell.hh"
#include "Obstacle.hh"
#include "Particle.hh"
#include "Polyhedron.hh"
#include "Quaternion.hh"
#include "ReaderXML.hh"
#include "AppPRSHydroFT.hh"
#include "RigidBodyWithCrust.hh"
#include "RawDataPostProcessingWriter.hh"
#include "SimpleObstacle.hh"
#include "Transform.hh"

namespace {

const double kPI = 3.14159265358979323846;

class OracleGrains : public Grains {
 public:
  AllComponents& comps() { return m_allcomponents; }
  LinkedCell* lc() { return m_collision; }
  void forces() { computeParticlesForceAndTorque(); }
  void move_only(double dtv, double dtx) {
    m_allcomponents.Move(m_time, dtv, dtx, dtx, m_collision);
  }
  void link_update() { m_collision->LinkUpdate(m_time, m_dt, m_allcomponents.getActiveParticles()); }
  void advance(double dtv) { m_allcomponents.advanceParticlesVelocity(m_time, dtv); }
  void kdk(double dt) {  // Grains::Simulation leapfrog branch (Grains.cpp:344-364)
    m_time += dt;
    moveParticlesAndObstacles(0.5 * dt, dt, dt);
    computeParticlesForceAndTorque();
    m_allcomponents.advanceParticlesVelocity(m_time, 0.5 * dt);
  }
  // the per-phase timers that Grains::Simulation registers (Grains.cpp:277-282)
  void register_timers() {
    SCT_insert_app("ParticlesInsertion");
    SCT_insert_app("ComputeForces");
    SCT_insert_app("Move");
    SCT_insert_app("UpdateParticleActivity");
    SCT_insert_app("LinkUpdate");
    SCT_insert_app("OutputResults");
  }
  double& time() { return m_time; }
  double& dt() { return m_dt; }
  // The collision App of this simulation replaced by `app`, as Grains::
  // Construction would register it in place of its LinkedCell (Grains.cpp:
  // 777-780): the first App of m_allApp and m_collision.  The stock LinkedCell
  // stays alive (its cells hold the particles' links) and is returned.
  LinkedCell* use_app(LinkedCell* app) {
    LinkedCell* old = m_collision;
    for (App*& a : m_allApp)
      if (a == old) a = app;
    m_collision = app;
    return old;
  }
  AllInsertionWindows const& windows() const { return m_insertion_windows; }
  // the fluid's hydrodynamic force App of GrainsCoupledWithFluid::Forces
  // (Fluid/src/GrainsCoupledWithFluid.cpp:455-462): registered after the
  // collision App, with arrays for the active particles
  AppPRSHydroFT* hydro_app() {
    if (!m_hydro) {
      m_hydro = new AppPRSHydroFT();
      m_hydro->setName("PRSHydroFT");
      m_allApp.push_back(m_hydro);
      m_hydro->allocateHydroFT(m_allcomponents.getActiveParticles()->size());
    }
    return m_hydro;
  }
  AppPRSHydroFT* m_hydro = nullptr;
};

struct ShapeSpec {
  int type;
  std::vector<double> p;
};

std::string num(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

}  // namespace

struct grains_gpu_ctx {
  grains_gpu_config cfg{};
  std::vector<ShapeSpec> shapes;
  grains_gpu_domain dom{};
  bool has_dom = false;
  std::map<std::pair<int, int>, std::pair<int, std::vector<double>>> laws;
  std::vector<grains_gpu_obstacle> obs;
  std::vector<grains_gpu_obstacle_loading> loads;  // explicit imposed motions
  int collision = GRAINS_GPU_GJK;                   // <CollisionDetection Type=...>
  double gjk_tol = 1e-10;                           // Tolerance=...
  int gjk_accel = 0, gjk_history = 0;               // Acceleration=..., History=...
  OracleGrains* g = nullptr;
  LinkedCell* stock_lc = nullptr;  // the reference's LinkedCell after grains_ref_use_gpu_app
  std::string dir;
  std::string err;
  int status = 0;
  std::vector<int> my_id;                // upload index -> my id
  std::map<int, Particle*> part_of_my;   // my id -> reference particle
  std::map<int, int> my_of_ref;          // reference id -> my id (particles and obstacles)
  std::map<int, int> ref_of_my;          // my id -> reference id
  std::set<int> obstacle_my_ids;
  std::vector<SimpleObstacle*> ref_obs;  // in definition order
  std::vector<std::pair<int, int>> last_contacts;
  long long steps = 0;
};

namespace {

int fail(grains_gpu_ctx* c, int code, const std::string& m) {
  c->err = m;
  c->status |= code;
  return code;
}

double sphere_volume(double r) { return 4.0 * kPI * std::pow(r, 3.) / 3.0; }

// a density giving exactly 'mass' for the shape volume (Particle.cpp:158)
double density_for(double mass, double vol) {
  double rho = mass / vol;
  for (int k = 0; k < 8 && rho * vol != mass; ++k) rho = std::nextafter(rho, rho * vol < mass ? 1e300 : -1e300);
  return rho;
}

// polyhedron file of the reference's format (Polyhedron::create,
// Geometry/src/Polyhedron.cpp:125-160, readFaces :374-408): dimension, vertex
// count, one vertex per line, a blank line, face count, then one face per line
// as its vertex indices only, without trailing blanks
std::string polyhedron_file(const std::string& dir, int shape, const ShapeSpec& s) {
  const std::string path = dir + "/poly" + std::to_string(shape) + ".txt";
  std::ofstream f(path.c_str());
  f.precision(17);
  const int nv = (int)s.p[0];
  f << "3\n" << nv << "\n";
  for (int v = 0; v < nv; ++v) f << s.p[1 + 3 * v] << " " << s.p[2 + 3 * v] << " " << s.p[3 + 3 * v] << "\n";
  size_t k = 1 + 3 * (size_t)nv;
  const int nf = (int)s.p[k++];
  f << "\n" << nf << "\n";
  for (int q = 0; q < nf; ++q) {
    const int m = (int)s.p[k++];
    for (int j = 0; j < m; ++j) f << (j ? " " : "") << (int)s.p[k++];
    f << "\n";
  }
  return path;
}

// the reference's own volume of a polyhedron file (Polyhedron::getVolume)
double polyhedron_volume(const std::string& dir, const std::string& path) {
  const std::string saved = GrainsExec::m_ReloadDirectory;
  GrainsExec::m_ReloadDirectory = dir;
  std::istringstream is(GrainsExec::extractFileName(path));
  Polyhedron* P = Polyhedron::create(is);
  GrainsExec::m_ReloadDirectory = saved;
  return P->getVolume();
}

void convex_xml(std::ostream& o, const ShapeSpec& s, double radius, const std::string& poly_path = "") {
  if (s.type == GRAINS_GPU_SPHERE) o << "<Sphere Radius=\"" << num(radius) << "\"/>";
  else if (s.type == GRAINS_GPU_POLYHEDRON) o << "<Polyhedron Name=\"" << poly_path << "\"/>";
  else if (s.type == GRAINS_GPU_BOX)
    o << "<Box LX=\"" << num(s.p[0]) << "\" LY=\"" << num(s.p[1]) << "\" LZ=\"" << num(s.p[2]) << "\"/>";
  else if (s.type == GRAINS_GPU_CYLINDER)
    o << "<Cylinder Radius=\"" << num(s.p[0]) << "\" Height=\"" << num(s.p[1]) << "\"/>";
}

void set_state(grains_gpu_ctx* c, Particle* P, const grains_gpu_particles* p, int64_t i) {
  double m[12];
  const double* q = p->quaternion + 4 * i;
  Quaternion qq(q[0], q[1], q[2], q[3]);
  if (p->basis) {
    for (int k = 0; k < 9; ++k) m[k] = p->basis[9 * i + k];
  } else {
    Transform const* t = P->getRigidBody()->getTransform();
    Matrix const& b = t->getBasis();
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) m[3 * r + cc] = b[r][cc];
  }
  // Component::setPosition(double const*) -> Transform::setValue: basis row
  // major (Matrix::setValue, Matrix.cpp:144-149) then origin
  double mm[12];
  for (int k = 0; k < 9; ++k) mm[k] = m[k];
  for (int k = 0; k < 3; ++k) mm[9 + k] = p->position[3 * i + k];
  P->setPosition(mm);
  P->setQuaternionRotation(qq);
  P->setTranslationalVelocity(Vector3(p->velocity[3 * i], p->velocity[3 * i + 1], p->velocity[3 * i + 2]));
  P->setAngularVelocity(Vector3(p->omega[3 * i], p->omega[3 * i + 1], p->omega[3 * i + 2]));
  P->initialize_transformWithCrust_to_notComputed();
}

}  // namespace

extern "C" {

int grains_ref_create(const grains_gpu_config* cfg, grains_gpu_ctx** out) {
  if (!cfg || !out || cfg->n_systems != 1) return GRAINS_GPU_INVALID_ARGUMENT;
  grains_gpu_ctx* c = new grains_gpu_ctx();
  c->cfg = *cfg;
  // the fluid settings are statics of Particle: back to the defaults
  // (Particle.cpp:21-23) for every new simulation
  Particle::setFluidDensity(0.);
  Particle::setFluidCorrectedAcceleration(true);
  char tmpl[] = "/tmp/grains_ref_XXXXXX";
  char* d = mkdtemp(tmpl);
  c->dir = d ? d : "/tmp";
  *out = c;
  return 0;
}

int grains_ref_destroy(grains_gpu_ctx* c) {
  if (!c) return 0;
  // The reference's Grains object is left alive on purpose: its destructor
  // deletes the contact-force models of ContactBuilderFactory's static table
  // without erasing them (ContactBuilderFactory.cpp:362-367, Grains.cpp:74),
  // and the next simulation built in this process would delete them again
  // when it defines its own (ContactBuilderFactory.cpp:107-108).  The next
  // simulation replaces the models; the old objects are never used again.
  c->g = nullptr;
  c->stock_lc = nullptr;
  std::string cmd = "rm -rf '" + c->dir + "'";
  if (c->dir.rfind("/tmp/grains_ref_", 0) == 0) (void)!system(cmd.c_str());
  delete c;
  return 0;
}

int grains_ref_last_error(const grains_gpu_ctx* c, char* buf, size_t len) {
  std::snprintf(buf, len, "%s", c->err.c_str());
  return 0;
}

int grains_ref_set_domain(grains_gpu_ctx* c, int32_t system, const grains_gpu_domain* d) {
  if (system != 0) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "one system only");
  c->dom = *d;
  c->has_dom = true;
  return 0;
}

int grains_ref_add_shape(grains_gpu_ctx* c, int32_t type, const double* p, int32_t n, int32_t* id) {
  c->shapes.push_back(ShapeSpec{type, std::vector<double>(p, p + n)});
  *id = (int)c->shapes.size() - 1;
  return 0;
}

int grains_ref_set_contact_law(grains_gpu_ctx* c, int32_t system, int32_t a, int32_t b, int32_t law,
                               const double* p, int32_t n) {
  c->laws[std::make_pair(std::min(a, b), std::max(a, b))] = std::make_pair(law, std::vector<double>(p, p + n));
  return 0;
}

int grains_ref_set_obstacles(grains_gpu_ctx* c, int32_t system, int32_t n, const grains_gpu_obstacle* o) {
  c->obs.assign(o, o + n);
  return 0;
}

int grains_ref_set_collision_algorithm(grains_gpu_ctx* c, int32_t algorithm) {
  if (algorithm != GRAINS_GPU_GJK && algorithm != GRAINS_GPU_GJK_SV) return GRAINS_GPU_INVALID_ARGUMENT;
  c->collision = algorithm;
  return 0;
}

int grains_ref_set_collision_options(grains_gpu_ctx* c, double tolerance, int32_t acceleration, int32_t history) {
  if (!(tolerance >= 1e-10) || (acceleration != 0 && acceleration != 1) || (history != 0 && history != 1))
    return GRAINS_GPU_INVALID_ARGUMENT;
  c->gjk_tol = tolerance;
  c->gjk_accel = acceleration;
  c->gjk_history = history;
  return 0;
}

// Particle::setFluidDensity / setFluidCorrectedAcceleration, then the
// weights and coupling factors of every particle (the reference's own
// computeWeight / setCouplingFactor; rho_p is each particle's class density)
int grains_ref_set_fluid(grains_gpu_ctx* c, double rho_f, int32_t corrected, const double* density) {
  (void)density;
  if (!c->g) return GRAINS_GPU_NOT_READY;
  Particle::setFluidDensity(rho_f);
  Particle::setFluidCorrectedAcceleration(corrected != 0);
  for (auto& kv : c->part_of_my) {
    kv.second->computeWeight();
    kv.second->setCouplingFactor();
  }
  return 0;
}

// AppPRSHydroFT::setHydroFT: its arrays follow the active particle list
int grains_ref_set_hydro_forces(grains_gpu_ctx* c, const double* force, const double* torque) {
  if (!c->g) return GRAINS_GPU_NOT_READY;
  std::map<Particle*, size_t> row;
  for (size_t i = 0; i < c->my_id.size(); ++i) row[c->part_of_my[c->my_id[i]]] = i;
  std::vector<std::vector<double>> h;
  for (Particle* P : *c->g->comps().getActiveParticles()) {
    if (P->getTag() >= 2) continue;
    std::vector<double> e(6, 0.);
    const size_t i = row[P];
    for (int k = 0; k < 3; ++k) {
      if (force) e[k] = force[3 * i + k];
      if (torque) e[3 + k] = torque[3 * i + k];
    }
    h.push_back(e);
  }
  c->g->hydro_app()->setHydroFT(&h);
  return 0;
}

// GrainsCoupledWithFluid::GrainsToFluid (Fluid/src/GrainsCoupledWithFluid.cpp:
// 912-1120) for the particles of this simulation, with the reference's own
// objects and number formatting, tokenised as GrainsToBasilisk does
// (InterfaceGrains3DBasilisk.cpp:64-87); particles by increasing id of the
// caller, indexed from 0
int grains_ref_fluid_features(grains_gpu_ctx* c, char* buf, int64_t cap, int64_t* len) {
  if (!c->g) return GRAINS_GPU_NOT_READY;
  auto D = [](double x) { return GrainsExec::doubleToString(ios::scientific, FORMAT16DIGITS, x); };
  ostringstream pf;
  pf << c->part_of_my.size() << endl;
  int k = 0;
  for (auto& kv : c->part_of_my) {
    Particle* P = kv.second;
    vector<double> inertia(6, 0.);
    P->computeInertiaTensorSpaceFixed(inertia);
    Matrix mr = P->getRigidBody()->getTransform()->getBasis();
    Vector3 const* vt = P->getTranslationalVelocity();
    Vector3 const* vr = P->getAngularVelocity();
    Point3 const* ce = P->getPosition();
    pf << k << " " << P->getNbCorners() << endl;
    pf << "P " << D((*vt)[X]) << " " << D((*vt)[Y]) << " " << D((*vt)[Z]) << " " << D((*vr)[X]) << " "
       << D((*vr)[Y]) << " " << D((*vr)[Z]) << " " << D(P->getDensity()) << " " << D(P->getMass());
    for (int t = 0; t < 6; ++t) pf << " " << D(inertia[t]);
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q) pf << " " << D(mr[r][q]);
    pf << " " << D((*ce)[X]) << " " << D((*ce)[Y]) << " " << D((*ce)[Z]) << endl;
    pf << P->getCircumscribedRadius();
    P->writePositionInFluid(pf);
    ++k;
  }
  istringstream iss(pf.str());
  std::string out, tok;
  while (iss >> tok) {
    out += tok;
    out += ' ';
  }
  *len = (int64_t)out.size() + 1;
  if (buf) {
    if (cap < *len) return GRAINS_GPU_INVALID_ARGUMENT;
    std::memcpy(buf, out.c_str(), out.size() + 1);
  }
  return 0;
}

int grains_ref_set_obstacle_loadings(grains_gpu_ctx* c, int32_t system, int32_t n,
                                     const grains_gpu_obstacle_loading* l) {
  (void)system;
  c->loads.assign(l, l + n);
  return 0;
}

int grains_ref_upload_particles(grains_gpu_ctx* c, const grains_gpu_particles* p) {
  if (!c->has_dom) return fail(c, GRAINS_GPU_NOT_READY, "no domain");
  if (c->g) return fail(c, GRAINS_GPU_NOT_READY, "one upload per context");
  const int64_t n = p->n;
  // particle classes: (shape, radius, crust, material, density)
  struct Cls {
    int shape;
    double radius, crust, rho;
    int material;
    std::vector<int64_t> members;
  };
  std::vector<Cls> classes;
  std::map<std::string, int> key_of;
  double rmax = 0;
  std::map<int, std::string> poly_path;
  std::map<int, double> poly_vol;
  for (size_t k = 0; k < c->shapes.size(); ++k)
    if (c->shapes[k].type == GRAINS_GPU_POLYHEDRON) {
      poly_path[(int)k] = polyhedron_file(c->dir, (int)k, c->shapes[k]);
      poly_vol[(int)k] = polyhedron_volume(c->dir, poly_path[(int)k]);
    }
  for (int64_t i = 0; i < n; ++i) {
    const ShapeSpec& s = c->shapes[p->shape[i]];
    double vol = s.type == GRAINS_GPU_SPHERE ? sphere_volume(p->radius[i])
                 : s.type == GRAINS_GPU_POLYHEDRON ? poly_vol[p->shape[i]]
                 : s.type == GRAINS_GPU_BOX ? s.p[0] * s.p[1] * s.p[2]
                                             : 2 * (s.p[1] / 2.) * kPI * s.p[0] * s.p[0];
    if (s.type == GRAINS_GPU_BOX) vol = 8.0 * (s.p[0] / 2.) * (s.p[1] / 2.) * (s.p[2] / 2.);
    double rho = density_for(p->mass[i], vol);
    std::string key = std::to_string(p->shape[i]) + "/" + num(p->radius[i]) + "/" + num(p->crust[i]) + "/" +
                      std::to_string(p->material[i]) + "/" + num(rho);
    auto it = key_of.find(key);
    if (it == key_of.end()) {
      key_of[key] = (int)classes.size();
      classes.push_back(Cls{p->shape[i], p->radius[i], p->crust[i], rho, p->material[i], {}});
      it = key_of.find(key);
    }
    classes[it->second].members.push_back(i);
    rmax = std::max(rmax, p->radius[i]);
  }
  // input file
  const grains_gpu_domain& d = c->dom;
  std::ostringstream x;
  x << "<Grains3D Type=\"Standard\">\n<Construction>\n";
  // the reference's domain is (origin, max corner) with size = max - origin
  // (App::set_dimensions, Base/src/App.cpp:35-53): a max corner whose
  // difference with the origin is exactly the requested size
  double mxyz[3];
  for (int a = 0; a < 3; ++a) {
    double m = d.origin[a] + d.size[a];
    for (int k = 0; k < 8 && m - d.origin[a] != d.size[a]; ++k)
      m = std::nextafter(m, m - d.origin[a] < d.size[a] ? 1e300 : -1e300);
    mxyz[a] = m;
  }
  // every attribute is written: the reference keeps them in GrainsExec
  // statics that only a present attribute sets (Grains.cpp:654-723), so a
  // simulation built after another in this process must restate the defaults
  x << "<CollisionDetectionAlgorithm><CollisionDetection Type=\""
    << (c->collision == GRAINS_GPU_GJK_SV ? "GJK_SV" : "GJK") << "\" Tolerance=\"" << num(c->gjk_tol)
    << "\" Acceleration=\"" << (c->gjk_accel ? "ON" : "OFF") << "\" History=\""
    << (c->gjk_history ? "ON" : "OFF") << "\"/></CollisionDetectionAlgorithm>\n";
  x << "<LinkedCell MX=\"" << num(mxyz[0]) << "\" MY=\"" << num(mxyz[1]) << "\" MZ=\"" << num(mxyz[2])
    << "\" CellSizeFactor=\"" << num(d.cell_size / (2. * rmax)) << "\"/>\n";
  x << "<Origin OX=\"" << num(d.origin[0]) << "\" OY=\"" << num(d.origin[1]) << "\" OZ=\"" << num(d.origin[2])
    << "\"/>\n<Periodicity PX=\"0\" PY=\"0\" PZ=\"0\"/>\n";
  x << "<ContactForceModels>\n";
  for (auto& kv : c->laws) {
    x << "<ContactForceModel><Material materialA=\"m" << kv.first.first << "\" materialB=\"m" << kv.first.second
      << "\"/>";
    const std::vector<double>& q = kv.second.second;
    if (kv.second.first == GRAINS_GPU_HOOKE_MEMORY) {
      x << "<HookeMemory><kn>" << num(q[0]) << "</kn><en>" << num(q[1]) << "</en><etat>" << num(q[2])
        << "</etat><muc>" << num(q[3]) << "</muc><kt>" << num(q[4]) << "</kt><mur>" << num(q[5]) << "</mur><etarpf>"
        << num(q[6]) << "</etarpf>";
      if (q[7] != 0.) x << "<epst>" << num(q[7]) << "</epst>";
      x << "</HookeMemory>";
    } else if (kv.second.first == GRAINS_GPU_HERTZ) {
      x << "<Hertz><Es>" << num(q[0]) << "</Es><en>" << num(q[1]) << "</en><muc>" << num(q[2]) << "</muc><kr>"
        << num(q[3]) << "</kr><Gs>" << num(q[4]) << "</Gs></Hertz>";
    } else if (kv.second.first == GRAINS_GPU_HERTZ_MEMORY) {
      x << "<HertzMemory><Es>" << num(q[0]) << "</Es><en>" << num(q[1]) << "</en><muc>" << num(q[2]) << "</muc><Gs>"
        << num(q[3]) << "</Gs><mur>" << num(q[4]) << "</mur><etarpf>" << num(q[5]) << "</etarpf>";
      if (q[6] != 0.) x << "<epst>" << num(q[6]) << "</epst>";
      x << "</HertzMemory>";
    } else {
      x << "<Hooke><kn>" << num(q[0]) << "</kn><en>" << num(q[1]) << "</en><etat>" << num(q[2]) << "</etat><muc>"
        << num(q[3]) << "</muc><kr>" << num(q[4]) << "</kr></Hooke>";
    }
    x << "</ContactForceModel>\n";
  }
  x << "</ContactForceModels>\n<Particles>\n";
  for (auto& k : classes) {
    x << "<Particle Number=\"" << k.members.size() << "\" Density=\"" << num(k.rho) << "\"><Convex CrustThickness=\""
      << num(k.crust) << "\">\n";
    convex_xml(x, c->shapes[k.shape], k.radius, poly_path.count(k.shape) ? poly_path[k.shape] : "");
    x << "\n</Convex><AngularPosition Type=\"Identity\"></AngularPosition><Material>m" << k.material
      << "</Material></Particle>\n";
  }
  x << "</Particles>\n<Obstacles>\n";
  for (size_t k = 0; k < c->obs.size(); ++k) {
    const grains_gpu_obstacle& o = c->obs[k];
    const ShapeSpec& s = c->shapes[o.shape];
    x << "<Obstacle name=\"o" << k << "\" Type=\"Standard\"><Convex CrustThickness=\"" << num(o.crust) << "\">\n";
    convex_xml(x, s, 0.);
    x << "\n</Convex><Centre X=\"" << num(o.transform[9]) << "\" Y=\"" << num(o.transform[10]) << "\" Z=\""
      << num(o.transform[11]) << "\"/>";
    bool identity = true;
    for (int q = 0; q < 9; ++q) identity = identity && o.transform[q] == (q % 4 == 0 ? 1. : 0.);
    if (identity) {
      x << "<AngularPosition Type=\"Identity\"></AngularPosition>";
    } else {  // row-major rotation matrix (Transform::load, Geometry/src/Transform.cpp:510-529)
      x << "<AngularPosition Type=\"Matrix\">";
      for (int q = 0; q < 9; ++q) x << (q ? " " : "") << num(o.transform[q]);
      x << "</AngularPosition>";
    }
    x << "<Material>m" << o.material << "</Material></Obstacle>\n";
  }
  x << "</Obstacles>\n</Construction>\n<Forces><Gravity GX=\"" << num(d.gravity[0]) << "\" GY=\"" << num(d.gravity[1])
    << "\" GZ=\"" << num(d.gravity[2]) << "\"/></Forces>\n";
  x << "<Simulation>\n<TimeInterval Start=\"0.\" End=\"1.e9\"/>\n<TimeStep dt=\"1.e-5\"/>\n";
  x << "<RestartFile Name=\"" << c->dir << "/restart\" WritingMode=\"Text\"/>\n";
  x << "<TimeSave Start=\"1.e8\" End=\"1.e9\" Every=\"1.e8\"/>\n";
  x << "<ParticleInsertion><Mode Type=\"InitialTime\"/><Order Type=\"Ordered\"/>"
       "<InitialAngularPosition Type=\"Fixed\"/><RandomGeneratorSeed Type=\"Default\"/><Frequency TryEvery=\"1\"/>"
       "<ForceInsertion Value=\"True\"/><ParticlePosition><File Name=\""
    << c->dir << "/positions.txt\"/></ParticlePosition></ParticleInsertion>\n";
  // imposed obstacle motion (Grains::AdditionalFeatures, Base/src/Grains.cpp:1719-1745;
  // ObstacleImposedVelocity.cpp:38-260): a constant rotation about the
  // obstacle's rotation centre, or a constant translation
  // explicit loadings (<ObstacleLoading> per motion, ObstacleImposedVelocity.cpp:60-262) replace an
  // obstacle's legacy motion fields
  auto has_explicit = [&](int id) {
    for (auto& l : c->loads)
      if (l.obstacle_id == id) return true;
    return false;
  };
  bool any_moving = !c->loads.empty();
  for (auto& o : c->obs) any_moving = any_moving || o.moving;
  if (any_moving) {
    x << "<ObstacleLoadings>\n";
    for (size_t k = 0; k < c->obs.size(); ++k) {
      const grains_gpu_obstacle& o = c->obs[k];
      if (!o.moving || has_explicit(o.id)) continue;
      x << "<ObstacleLoading Type=\"Velocity\" ObstacleName=\"o" << k
        << "\"><TimeInterval Start=\"0.\" End=\"1.e9\"/>";
      if (o.omega[0] != 0. || o.omega[1] != 0. || o.omega[2] != 0.)
        x << "<ConstantRotation><AngularVelocity WX=\"" << num(o.omega[0]) << "\" WY=\"" << num(o.omega[1])
          << "\" WZ=\"" << num(o.omega[2]) << "\"/><RotationCenter CX=\"" << num(o.rotation_center[0]) << "\" CY=\""
          << num(o.rotation_center[1]) << "\" CZ=\"" << num(o.rotation_center[2]) << "\"/></ConstantRotation>";
      else
        x << "<ConstantTranslation><TranslationalVelocity VX=\"" << num(o.velocity[0]) << "\" VY=\""
          << num(o.velocity[1]) << "\" VZ=\"" << num(o.velocity[2]) << "\"/></ConstantTranslation>";
      x << "</ObstacleLoading>\n";
    }
    for (const auto& l : c->loads) {
      size_t k = 0;
      while (k < c->obs.size() && c->obs[k].id != l.obstacle_id) ++k;
      if (k == c->obs.size()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "loading of an unknown obstacle");
      // Type="Force": ObstacleImposedForce (Grains.cpp:1736-1742, ObstacleImposedForce.cpp:29-80)
      x << "<ObstacleLoading Type=\"" << (l.type == GRAINS_GPU_FORCE_TRANSLATION ? "Force" : "Velocity")
        << "\" ObstacleName=\"o" << k << "\"><TimeInterval Start=\"" << num(l.t_start) << "\" End=\""
        << num(l.t_end) << "\"/>";
      auto vec = [&](const char* tag, const char* a, const char* b, const char* cc, const double* v) {
        x << "<" << tag << " " << a << "=\"" << num(v[0]) << "\" " << b << "=\"" << num(v[1]) << "\" " << cc
          << "=\"" << num(v[2]) << "\"/>";
      };
      switch (l.type) {
        case GRAINS_GPU_CONSTANT_TRANSLATION:
          x << "<ConstantTranslation>";
          vec("TranslationalVelocity", "VX", "VY", "VZ", l.vector);
          x << "</ConstantTranslation>";
          break;
        case GRAINS_GPU_SIN_TRANSLATION:
        case GRAINS_GPU_CRENEL_TRANSLATION:
          x << (l.type == GRAINS_GPU_SIN_TRANSLATION ? "<SinTranslation>" : "<CrenelTranslation>");
          vec("Direction", "VX", "VY", "VZ", l.vector);
          x << "<Parameters Amplitude=\"" << num(l.amplitude[0]) << "\" Period=\"" << num(l.period[0]) << "\"";
          if (l.type == GRAINS_GPU_SIN_TRANSLATION) x << " PhaseShift=\"" << num(l.phase_deg[0]) << "\"";
          x << "/>" << (l.type == GRAINS_GPU_SIN_TRANSLATION ? "</SinTranslation>" : "</CrenelTranslation>");
          break;
        case GRAINS_GPU_CONSTANT_ROTATION:
          x << "<ConstantRotation>";
          vec("AngularVelocity", "WX", "WY", "WZ", l.vector);
          if (l.has_center) vec("RotationCenter", "CX", "CY", "CZ", l.center);
          x << "</ConstantRotation>";
          break;
        case GRAINS_GPU_MULTISIN_TRANSLATION:
          x << "<MultiSinTranslation>";
          vec("Direction", "VX", "VY", "VZ", l.vector);
          vec("Period", "PX", "PY", "PZ", l.period);
          vec("PhaseShift", "PhiX", "PhiY", "PhiZ", l.phase_deg);
          vec("Amplitude", "AX", "AY", "AZ", l.amplitude);
          x << "</MultiSinTranslation>";
          break;
        case GRAINS_GPU_FORCE_TRANSLATION:
          x << "<ConstantTranslation>";
          vec("Amplitude", "AX", "AY", "AZ", l.vector);
          x << "<Property ";
          if (l.amplitude[0] > 0.) x << "Mass=\"" << num(l.amplitude[0]) << "\" ";
          x << "Vmax=\"" << num(l.amplitude[1]) << "\"/></ConstantTranslation>";
          break;
        default:
          return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "unknown loading type");
      }
      x << "</ObstacleLoading>\n";
    }
    x << "</ObstacleLoadings>\n";
  }
  x << "</Simulation>\n</Grains3D>\n";
  {
    std::ofstream f((c->dir + "/input.xml").c_str());
    f << x.str();
    std::ofstream fp((c->dir + "/positions.txt").c_str());
    fp.precision(17);
    for (auto& k : classes)
      for (int64_t i : k.members)
        fp << p->position[3 * i] << " " << p->position[3 * i + 1] << " " << p->position[3 * i + 2] << "\n";
  }
  // build the simulation
  std::streambuf* old = std::cout.rdbuf();
  std::ofstream log((c->dir + "/grains.log").c_str());
  std::cout.rdbuf(log.rdbuf());
  ReaderXML::initialize();
  DOMElement* root = ReaderXML::getRoot(c->dir + "/input.xml");
  GrainsBuilderFactory::create(root);  // sets the 3D context
  c->g = new OracleGrains();
  c->g->do_before_time_stepping(root);
  c->g->register_timers();
  std::cout.rdbuf(old);
  // match reference particles to uploaded ones by insertion position
  std::map<std::vector<double>, int64_t> by_pos;
  for (int64_t i = 0; i < n; ++i)
    by_pos[std::vector<double>(p->position + 3 * i, p->position + 3 * i + 3)] = i;
  c->my_id.assign(p->id, p->id + n);
  for (Particle* P : *c->g->comps().getActiveParticles()) {
    Point3 const* o = P->getPosition();
    auto it = by_pos.find(std::vector<double>{(*o)[0], (*o)[1], (*o)[2]});
    if (it == by_pos.end()) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "reference particle not matched");
    int my = p->id[it->second];
    c->part_of_my[my] = P;
    c->my_of_ref[P->getID()] = my;
    c->ref_of_my[my] = P->getID();
  }
  if ((int64_t)c->part_of_my.size() != n) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "particle count mismatch");
  std::list<SimpleObstacle*> ol = c->g->comps().getObstacles()->getObstacles();
  for (SimpleObstacle* o : ol) c->ref_obs.push_back(o);
  for (size_t k = 0; k < c->ref_obs.size() && k < c->obs.size(); ++k) {
    c->my_of_ref[c->ref_obs[k]->getID()] = c->obs[k].id;
    c->ref_of_my[c->obs[k].id] = c->ref_obs[k]->getID();
    c->obstacle_my_ids.insert(c->obs[k].id);
  }
  // overwrite the kinematic state with the uploaded one, clear memories, relink
  for (int64_t i = 0; i < n; ++i) set_state(c, c->part_of_my[p->id[i]], p, i);
  for (Particle* P : *c->g->comps().getActiveParticles()) {
    auto* cm = const_cast<std::map<std::tuple<int, int, int>, std::tuple<bool, Vector3, Vector3, Vector3>>*>(
        P->getContactMap());
    cm->clear();
  }
  for (SimpleObstacle* o : c->ref_obs) {
    auto* cm = const_cast<std::map<std::tuple<int, int, int>, std::tuple<bool, Vector3, Vector3, Vector3>>*>(
        o->getContactMap());
    cm->clear();
  }
  c->g->link_update();
  return 0;
}

int grains_ref_update_particles(grains_gpu_ctx* c, const grains_gpu_particles* p) {
  for (int64_t i = 0; i < p->n; ++i) set_state(c, c->part_of_my[c->my_id[i]], p, i);
  c->g->link_update();
  return 0;
}

int grains_ref_download_particles(grains_gpu_ctx* c, grains_gpu_particles* p) {
  int64_t n = std::min<int64_t>(p->n, (int64_t)c->my_id.size());
  for (int64_t i = 0; i < n; ++i) {
    Particle* P = c->part_of_my[c->my_id[i]];
    if (p->id) p->id[i] = c->my_id[i];
    auto put = [&](double* a, Vector3 const& v) {
      if (a) for (int k = 0; k < 3; ++k) a[3 * i + k] = v[k];
    };
    Point3 const* o = P->getPosition();
    if (p->position) for (int k = 0; k < 3; ++k) p->position[3 * i + k] = (*o)[k];
    put(p->velocity, *P->getTranslationalVelocity());
    put(p->omega, *P->getAngularVelocity());
    put(p->force, *P->getForce());
    put(p->torque, *P->getTorque());
    if (p->quaternion) {
      Quaternion const* q = P->getQuaternionRotation();
      for (int k = 0; k < 4; ++k) p->quaternion[4 * i + k] = (*q)[k];
    }
    if (p->basis) {
      Matrix const& b = P->getRigidBody()->getTransform()->getBasis();
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) p->basis[9 * i + 3 * r + cc] = b[r][cc];
    }
    if (p->coordination) p->coordination[i] = P->getCoordinationNumber();
  }
  p->n = n;
  return 0;
}

int grains_ref_upload_contact_memory(grains_gpu_ctx* c, const grains_gpu_contact_memory* m) {
  for (int64_t k = 0; k < m->n; ++k) {
    auto io = c->ref_of_my.find(m->owner[k]);
    auto it = c->ref_of_my.find(m->other[k]);
    if (io == c->ref_of_my.end() || it == c->ref_of_my.end()) continue;
    Component* owner = nullptr;
    if (c->obstacle_my_ids.count(m->owner[k])) {
      for (size_t q = 0; q < c->obs.size(); ++q)
        if (c->obs[q].id == m->owner[k]) owner = c->ref_obs[q];
    } else {
      owner = c->part_of_my[m->owner[k]];
    }
    if (!owner) continue;
    owner->copyContactInMap(std::make_tuple(1, it->second, 1), true,
                            Vector3(m->kdelta[3 * k], m->kdelta[3 * k + 1], m->kdelta[3 * k + 2]),
                            Vector3(m->prev_normal[3 * k], m->prev_normal[3 * k + 1], m->prev_normal[3 * k + 2]),
                            Vector3(m->spring_torque[3 * k], m->spring_torque[3 * k + 1], m->spring_torque[3 * k + 2]));
  }
  return 0;
}

int grains_ref_download_contact_memory(grains_gpu_ctx* c, grains_gpu_contact_memory* m) {
  int64_t k = 0, cap = m->n;
  std::vector<std::pair<int, Component*>> comps;
  for (int my : c->my_id) comps.push_back(std::make_pair(my, (Component*)c->part_of_my[my]));
  for (size_t q = 0; q < c->ref_obs.size(); ++q) comps.push_back(std::make_pair(c->obs[q].id, (Component*)c->ref_obs[q]));
  for (auto& pc : comps)
    for (auto& kv : *pc.second->getContactMap()) {
      if (k < cap) {
        m->owner[k] = pc.first;
        m->other[k] = c->my_of_ref[std::get<1>(kv.first)];
        Vector3 const* v[3] = {&std::get<1>(kv.second), &std::get<2>(kv.second), &std::get<3>(kv.second)};
        double* dst[3] = {m->kdelta, m->prev_normal, m->spring_torque};
        for (int t = 0; t < 3; ++t)
          for (int a = 0; a < 3; ++a) dst[t][3 * k + a] = (*v[t])[a];
      }
      ++k;
    }
  m->n = k;
  return k > cap ? GRAINS_GPU_PAIR_OVERFLOW : 0;
}

int grains_ref_download_obstacles(grains_gpu_ctx* c, int32_t system, int32_t n, double* t) {
  for (int i = 0; i < n && i < (int)c->ref_obs.size(); ++i) {
    Transform const* tr = c->ref_obs[i]->getRigidBody()->getTransform();
    Matrix const& b = tr->getBasis();
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) t[12 * i + 3 * r + cc] = b[r][cc];
    Point3 const* o = tr->getOrigin();
    for (int k = 0; k < 3; ++k) t[12 * i + 9 + k] = (*o)[k];
  }
  return 0;
}

static void record_contacts(grains_gpu_ctx* c) {
  c->last_contacts.clear();
  for (int my : c->my_id) {
    Particle* P = c->part_of_my[my];
    for (auto& kv : *P->getContactMap()) {
      int other = c->my_of_ref[std::get<1>(kv.first)];
      if (c->obstacle_my_ids.count(other)) continue;
      if (my < other) c->last_contacts.push_back(std::make_pair(my, other));
    }
  }
}

static int guarded(grains_gpu_ctx* c, void (*fn)(grains_gpu_ctx*, double, double), double a, double b) {
  std::streambuf* old = std::cout.rdbuf();
  std::ofstream log((c->dir + "/grains.log").c_str(), std::ios::app);
  std::cout.rdbuf(log.rdbuf());
  int rc = 0;
  try {
    fn(c, a, b);
  } catch (ContactError&) {
    rc = fail(c, GRAINS_GPU_CONTACT_ERROR, "ContactError");
  } catch (MotionError&) {
    rc = fail(c, GRAINS_GPU_MOTION_ERROR, "MotionError");
  } catch (SimulationError&) {
    rc = fail(c, GRAINS_GPU_OUT_OF_GRID, "SimulationError");
  }
  std::cout.rdbuf(old);
  return rc;
}

// The reference's own time loop with the B200 collision App: LinkedCellGPU
// takes the place of the reference's LinkedCell in this simulation (as
// Grains::Construction registers its LinkedCell, Grains.cpp:777-780).  gpu_ctx:
// a grains_gpu context holding the same particles in the same upload order,
// with the same shapes, laws and walls.
int grains_ref_use_gpu_app(grains_gpu_ctx* c, void* gpu_ctx) {
  if (!c || !c->g || !gpu_ctx || c->stock_lc) return GRAINS_GPU_INVALID_ARGUMENT;
  LinkedCellGPU* app = new LinkedCellGPU(static_cast<grains_gpu_ctx*>(gpu_ctx));
  std::map<int, int> row_of_my, rows;
  for (size_t i = 0; i < c->my_id.size(); ++i) row_of_my[c->my_id[i]] = (int)i;
  for (auto& kv : c->my_of_ref)
    if (row_of_my.count(kv.second)) rows[kv.first] = row_of_my[kv.second];
  app->setRows(rows);
  app->setName("LinkedCell");
  c->stock_lc = c->g->use_app(app);
  return 0;
}

int grains_ref_compute_forces(grains_gpu_ctx* c, double time, double dt) {
  c->g->dt() = dt;
  int rc = guarded(c, [](grains_gpu_ctx* cc, double, double) { cc->g->forces(); }, 0, 0);
  record_contacts(c);
  return rc;
}

int grains_ref_move(grains_gpu_ctx* c, double time, double dt_v, double dt_x) {
  return guarded(c, [](grains_gpu_ctx* cc, double a, double b) { cc->g->move_only(a, b); }, dt_v, dt_x);
}

int grains_ref_link_update(grains_gpu_ctx* c, double time, double dt) {
  return guarded(c, [](grains_gpu_ctx* cc, double, double) { cc->g->link_update(); }, 0, 0);
}

int grains_ref_advance_velocity(grains_gpu_ctx* c, double time, double dt_v) {
  return guarded(c, [](grains_gpu_ctx* cc, double a, double) { cc->g->advance(a); }, dt_v, 0);
}

int grains_ref_initialize_leapfrog(grains_gpu_ctx* c, double time, double dt) {
  if (int rc = grains_ref_compute_forces(c, time, dt)) return rc;
  c->g->comps().setAllContactMapCumulativeFeaturesToZero();
  return 0;
}

int grains_ref_step(grains_gpu_ctx* c, int32_t n, double* time, double dt) {
  c->g->dt() = dt;
  c->g->time() = *time;
  for (int k = 0; k < n; ++k) {
    int rc = guarded(c, [](grains_gpu_ctx* cc, double a, double) { cc->g->kdk(a); }, dt, 0);
    if (rc) return rc;
    *time += dt;
    c->steps++;
  }
  record_contacts(c);
  return 0;
}

int grains_ref_get_candidate_pairs(grains_gpu_ctx* c, int32_t system, int32_t include_obstacles, int64_t cap,
                                   int32_t* pairs, int64_t* n) {
  // cells of the reference's linked-cell assignment (Particle::getCell / Cell::getID)
  LinkedCell* lc = c->g->lc();
  double cs[3] = {lc->getCellSize(0), lc->getCellSize(1), lc->getCellSize(2)};
  int nb[3];
  for (int a = 0; a < 3; ++a) nb[a] = (int)std::lround(c->dom.size[a] / cs[a]);
  std::vector<std::pair<int, int>> out;
  std::vector<std::vector<int>> ijk;
  std::vector<int> ids;
  for (int my : c->my_id) {
    int id = c->part_of_my[my]->getCell()->getID();
    int i = id % nb[0], k = (id / nb[0]) % nb[2], j = id / (nb[0] * nb[2]);
    ijk.push_back({i, j, k});
    ids.push_back(my);
  }
  for (size_t a = 0; a < ids.size(); ++a)
    for (size_t b = a + 1; b < ids.size(); ++b)
      if (std::abs(ijk[a][0] - ijk[b][0]) <= 1 && std::abs(ijk[a][1] - ijk[b][1]) <= 1 &&
          std::abs(ijk[a][2] - ijk[b][2]) <= 1)
        out.push_back(std::make_pair(std::min(ids[a], ids[b]), std::max(ids[a], ids[b])));
  std::sort(out.begin(), out.end());
  *n = (int64_t)out.size();
  for (int64_t k = 0; k < *n && k < cap; ++k) {
    pairs[2 * k] = out[k].first;
    pairs[2 * k + 1] = out[k].second;
  }
  return *n > cap ? GRAINS_GPU_PAIR_OVERFLOW : 0;
}

int grains_ref_get_contact_pairs(grains_gpu_ctx* c, int32_t system, int64_t cap, int32_t* pairs, int64_t* n) {
  std::vector<std::pair<int, int>> out = c->last_contacts;
  std::sort(out.begin(), out.end());
  *n = (int64_t)out.size();
  for (int64_t k = 0; k < *n && k < cap; ++k) {
    pairs[2 * k] = out[k].first;
    pairs[2 * k + 1] = out[k].second;
  }
  return *n > cap ? GRAINS_GPU_PAIR_OVERFLOW : 0;
}

int grains_ref_get_stats(grains_gpu_ctx* c, grains_gpu_stats* st) {
  std::memset(st, 0, sizeof(*st));
  st->n_particles = (int64_t)c->my_id.size();
  int64_t nc = 0, no = 0;
  for (int my : c->my_id)
    for (auto& kv : *c->part_of_my[my]->getContactMap()) {
      int other = c->my_of_ref[std::get<1>(kv.first)];
      if (c->obstacle_my_ids.count(other)) ++no;
      else if (my < other) ++nc;
    }
  st->n_contacts = nc;
  st->n_obstacle_contacts = no;
  st->n_steps_done = c->steps;
  st->status = c->status;
  // the reference's own running statistics (AppCollision.cpp:160-187); they
  // run over the whole simulation (reset_stats does not clear them)
  st->overlap_max = c->g->lc()->getOverlapMax();
  st->overlap_mean = c->g->lc()->getOverlapMean();
  st->gjk_iterations_mean = c->g->lc()->getNbIterGJKMean();
  return 0;
}

int grains_ref_reset_stats(grains_gpu_ctx* c) {
  c->status = 0;
  return 0;
}

// The reference's own writers on the reference state, for the I/O fixtures:
// AllComponents::write (AllComponents.cpp:1062-1181) writes the particle file
// <root>_Particles.result (".bin" appended in Hybrid mode), moved to `path`.
int grains_ref_write_reload_particles(grains_gpu_ctx* c, const char* path, int32_t binary, int64_t* bytes) {
  if (!c || !c->g || !path) return GRAINS_GPU_INVALID_ARGUMENT;
  const std::string root = c->dir + "/refsave";
  GrainsExec::m_writingModeHybrid = binary != 0;
  std::ostringstream head;
  std::vector<Point3> known;
  c->g->comps().write(head, root + ".x", &known, CIR_NONE, c->g->lc(), 0, 1, nullptr);
  GrainsExec::m_writingModeHybrid = false;
  const std::string pfile = root + "_Particles.result" + (binary ? ".bin" : "");
  if (std::rename(pfile.c_str(), path) != 0) return fail(c, GRAINS_GPU_INVALID_ARGUMENT, "cannot move " + pfile);
  if (bytes) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    *bytes = (int64_t)f.tellg();
  }
  return 0;
}

// RawDataPostProcessingWriter (PostProcessing/src/RawDataPostProcessingWriter.cpp)
// for one output time: a writer built from <RawData Name=root WritingMode=...>,
// started in "new" mode (truncating) or appending, then closed.  The
// reference numbers the columns 1..GrainsExec::getTotalNumberPhysicalParticles
// itself; n_total is not used.
int grains_ref_write_rawdata(grains_gpu_ctx* c, const char* root, double time, int32_t system, int32_t n_total,
                             int32_t binary, int32_t truncate, int64_t* bytes) {
  (void)system;
  (void)n_total;
  if (!c || !c->g || !root) return GRAINS_GPU_INVALID_ARGUMENT;
  const std::string xml = c->dir + "/rawdata.xml";
  {
    std::ofstream f(xml.c_str());
    f << "<RawData Name=\"" << root << "\" WritingMode=\"" << (binary ? "Binary" : "Text") << "\"/>\n";
  }
  DOMElement* node = ReaderXML::getRoot(xml);
  const std::string saved = GrainsExec::m_ReloadType;
  GrainsExec::m_ReloadType = truncate ? "new" : "same";
  std::streambuf* old = std::cout.rdbuf();
  std::ostringstream quiet;
  std::cout.rdbuf(quiet.rdbuf());
  RawDataPostProcessingWriter* w = new RawDataPostProcessingWriter(node, 0, 1, false);
  AllComponents& a = c->g->comps();
  w->PostProcessing_start(time, c->g->dt(), a.getActiveParticles(), nullptr, nullptr, a.getReferenceParticles(),
                          a.getObstacles(), c->g->lc(), c->g->windows());
  w->PostProcessing_end();
  delete w;
  std::cout.rdbuf(old);
  GrainsExec::m_ReloadType = saved;
  if (bytes) *bytes = 0;
  return 0;
}

}  // extern "C"
