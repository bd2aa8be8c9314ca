"""ctypes binding of the C ABI in include/grains_gpu.h.

`GrainsLib` loads a shared library that exports the grains_gpu entry points
(or the same set under another prefix) and `Simulation` wraps one context with
numpy arrays.  Errors raise the Python counterparts of the reference's C++
exceptions (Grains/Base/include/Error.hh): ContactError, MotionError,
SimulationError.
"""
import ctypes as C
import os

import numpy as np

# ---- status bits (include/grains_gpu.h) ----------------------------------------
OK = 0
CONTACT_ERROR = 1 << 0
MOTION_ERROR = 1 << 1
OUT_OF_GRID = 1 << 2
PAIR_OVERFLOW = 1 << 3
HISTORY_FULL = 1 << 4
CUDA_ERROR = 1 << 5
TIMEOUT = 1 << 6
INVALID_ARGUMENT = 1 << 7
NOT_READY = 1 << 8
GJK_NOT_CONVERGED = 1 << 9
CONTACT_HANDLED = 1 << 10
CELL_TOO_SMALL = 1 << 11

FP64 = 0
MIXED = 1

SPHERE, BOX, CYLINDER, POLYHEDRON = 0, 1, 2, 3
GJK, GJK_SV = 0, 1
HOOKE, HOOKE_MEMORY, HERTZ, HERTZ_MEMORY = 0, 1, 2, 3


class GrainsError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("status 0x%x: %s" % (code, message))
        self.code = code


class ContactError(GrainsError):
    """Overlap reached the crust sum (RigidBodyWithCrust.cpp:620-629)."""


class MotionError(GrainsError):
    """Displacement over one step larger than the crust (Particle.cpp:447-457)."""


class SimulationError(GrainsError):
    """A particle left the linked-cell grid (LinkedCell.cpp:1525-1531)."""


def error_for(code, message):
    if code & CONTACT_ERROR:
        return ContactError(code, message)
    if code & MOTION_ERROR:
        return MotionError(code, message)
    if code & OUT_OF_GRID:
        return SimulationError(code, message)
    return GrainsError(code, message)


# ---- structures --------------------------------------------------------------
class Config(C.Structure):
    _fields_ = [("precision", C.c_int32), ("device", C.c_int32), ("n_systems", C.c_int32),
                ("history_capacity", C.c_int32), ("max_particles", C.c_int64), ("max_obstacles", C.c_int32),
                ("max_shapes", C.c_int32), ("max_materials", C.c_int32), ("reserved", C.c_int32 * 7)]


class Domain(C.Structure):
    _fields_ = [("origin", C.c_double * 3), ("size", C.c_double * 3), ("cell_size", C.c_double),
                ("gravity", C.c_double * 3)]


class Obstacle(C.Structure):
    _fields_ = [("id", C.c_int32), ("shape", C.c_int32), ("material", C.c_int32), ("moving", C.c_int32),
                ("crust", C.c_double), ("transform", C.c_double * 12), ("velocity", C.c_double * 3),
                ("omega", C.c_double * 3), ("rotation_center", C.c_double * 3)]


class ObstacleLoading(C.Structure):
    _fields_ = [("obstacle_id", C.c_int32), ("type", C.c_int32), ("t_start", C.c_double), ("t_end", C.c_double),
                ("vector", C.c_double * 3), ("center", C.c_double * 3), ("has_center", C.c_int32),
                ("reserved", C.c_int32), ("amplitude", C.c_double * 3), ("period", C.c_double * 3),
                ("phase_deg", C.c_double * 3)]


# imposed obstacle motions (grains_gpu_motion)
CONSTANT_TRANSLATION, SIN_TRANSLATION, CRENEL_TRANSLATION, CONSTANT_ROTATION, MULTISIN_TRANSLATION = 0, 1, 2, 3, 4
FORCE_TRANSLATION = 5  # an imposed force (ObstacleImposedForce): vector = force, amplitude = (mass, Vmax)

_P_I32 = C.POINTER(C.c_int32)
_P_F64 = C.POINTER(C.c_double)


class Tuning(C.Structure):
    _fields_ = [("cell_factor", C.c_double), ("contacts_block", C.c_int32), ("forces_block", C.c_int32),
                ("list_capacity", C.c_int32), ("gather_every", C.c_int32), ("persistent", C.c_int32),
                ("reserved", C.c_int32 * 3)]


class Particles(C.Structure):
    _fields_ = [("n", C.c_int64), ("id", _P_I32), ("system", _P_I32), ("shape", _P_I32), ("material", _P_I32),
                ("radius", _P_F64), ("crust", _P_F64), ("mass", _P_F64), ("inertia", _P_F64),
                ("position", _P_F64), ("quaternion", _P_F64), ("basis", _P_F64), ("velocity", _P_F64),
                ("omega", _P_F64), ("force", _P_F64), ("torque", _P_F64), ("coordination", _P_I32)]


class ContactMemory(C.Structure):
    _fields_ = [("n", C.c_int64), ("owner", _P_I32), ("other", _P_I32), ("kdelta", _P_F64),
                ("prev_normal", _P_F64), ("spring_torque", _P_F64), ("system", _P_I32)]


class Stats(C.Structure):
    _fields_ = [("n_particles", C.c_int64), ("n_candidate_pairs", C.c_int64),
                ("n_obstacle_candidates", C.c_int64), ("n_contacts", C.c_int64),
                ("n_obstacle_contacts", C.c_int64), ("n_gjk_calls", C.c_int64), ("n_gjk_iterations", C.c_int64),
                ("overlap_max", C.c_double), ("overlap_sum", C.c_double), ("n_steps_done", C.c_int64),
                ("status", C.c_int32), ("reserved", C.c_int32), ("overlap_mean", C.c_double),
                ("gjk_iterations_mean", C.c_double)]


_VP = C.c_void_p
_SIGS = {
    "create": [C.POINTER(Config), C.POINTER(_VP)],
    "destroy": [_VP],
    "last_error": [_VP, C.c_char_p, C.c_size_t],
    "set_domain": [_VP, C.c_int32, C.POINTER(Domain)],
    "add_shape": [_VP, C.c_int32, _P_F64, C.c_int32, _P_I32],
    "set_contact_law": [_VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P_F64, C.c_int32],
    "set_obstacles": [_VP, C.c_int32, C.c_int32, C.POINTER(Obstacle)],
    "set_obstacle_loadings": [_VP, C.c_int32, C.c_int32, C.POINTER(ObstacleLoading)],
    "set_collision_algorithm": [_VP, C.c_int32],
    "set_collision_options": [_VP, C.c_double, C.c_int32, C.c_int32],
    "update_particle_rows": [_VP, C.c_int64, C.POINTER(C.c_int64), C.c_void_p],
    "set_fluid": [_VP, C.c_double, C.c_int32, _P_F64],
    "set_hydro_forces": [_VP, _P_F64, _P_F64],
    "set_velocities": [_VP, _P_F64, _P_F64],
    "fluid_step": [_VP, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_int64), C.POINTER(C.c_double)],
    "fluid_features": [_VP, C.c_char_p, C.c_int64, C.POINTER(C.c_int64)],
    "upload_particles": [_VP, C.POINTER(Particles)],
    "download_particles": [_VP, C.POINTER(Particles)],
    "update_particles": [_VP, C.POINTER(Particles)],
    "upload_contact_memory": [_VP, C.POINTER(ContactMemory)],
    "download_contact_memory": [_VP, C.POINTER(ContactMemory)],
    "download_obstacles": [_VP, C.c_int32, C.c_int32, _P_F64],
    "compute_forces": [_VP, C.c_double, C.c_double],
    "move": [_VP, C.c_double, C.c_double, C.c_double],
    "link_update": [_VP, C.c_double, C.c_double],
    "advance_velocity": [_VP, C.c_double, C.c_double],
    "initialize_leapfrog": [_VP, C.c_double, C.c_double],
    "step": [_VP, C.c_int32, _P_F64, C.c_double],
    "get_candidate_pairs": [_VP, C.c_int32, C.c_int32, C.c_int64, _P_I32, C.POINTER(C.c_int64)],
    "get_contact_pairs": [_VP, C.c_int32, C.c_int64, _P_I32, C.POINTER(C.c_int64)],
    "get_contact_forces": [_VP, C.c_int32, C.c_int64, _P_I32, _P_F64, C.POINTER(C.c_int64)],
    "get_stats": [_VP, C.POINTER(Stats)],
    "reset_stats": [_VP],
    "set_record_attributes": [_VP, C.c_int64, _P_I32, _P_I32, _P_I32, _P_I32],
    "write_reload_particles": [_VP, C.c_char_p, C.c_int32, C.POINTER(C.c_int64)],
    "write_rawdata": [_VP, C.c_char_p, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                      C.POINTER(C.c_int64)],
}
# diagnostics that the reference built from its sources (oracle/_ref) lacks
_OPTIONAL = {"get_contact_forces", "set_record_attributes", "set_collision_options", "update_particle_rows",
             "set_fluid", "set_hydro_forces", "set_velocities", "fluid_step", "fluid_features"}
_GPU_ONLY = {
    "get_stream": [_VP, C.POINTER(_VP)],
    "synchronize": [_VP],
    "launches_per_step": [_VP, C.POINTER(C.c_int64)],
    "set_barrier_test": [_VP, C.c_int64, C.c_int32],
    "profile_kernels": [_VP, C.c_int32, _P_F64, C.c_double, C.c_char_p, C.c_size_t, _P_F64,
                        C.POINTER(C.c_int64), C.c_int32, _P_I32],
    "shape_properties": [C.c_int32, _P_F64, C.c_int32, _P_F64, _P_F64, _P_F64],
    "get_tuning": [_VP, C.POINTER(Tuning)],
    "set_tuning": [_VP, C.POINTER(Tuning)],
    "autotune": [_VP, C.c_double, C.c_double, C.c_int32, C.POINTER(Tuning), _P_F64],
    "adjoint_create": [_VP, C.c_int32, C.POINTER(_VP)],
    "adjoint_destroy": [_VP],
    "adjoint_last_error": [_VP, C.c_char_p, C.c_size_t],
    "adjoint_law_slots": [_VP, _P_I32],
    "adjoint_forward": [_VP, C.c_int32, C.c_double, _P_F64, _P_F64, _P_F64],
    "adjoint_contact_signature": [_VP, C.POINTER(C.c_uint64), C.POINTER(C.c_int64)],
    "adjoint_backward": [_VP, _P_F64, _P_F64, _P_F64, _P_F64, _P_F64, _P_F64, _P_F64, C.c_int32],
    "reload_open": [C.c_char_p, C.c_int32, C.POINTER(_VP)],
    "reload_last_error": [_VP, C.c_char_p, C.c_size_t],
    "reload_get": [_VP, C.c_void_p],
    "reload_close": [_VP],
    "format_double": [C.c_double, C.c_int32, C.c_char_p, C.c_size_t, _P_I32],
    "format_doubles": [_P_F64, C.c_int64, C.c_int32, C.c_char_p, C.c_int64, C.POINTER(C.c_int64)],
}


class ReloadData(C.Structure):
    _fields_ = [("n_particles", C.c_int64), ("n_memory", C.c_int64), ("geom_type", _P_I32), ("id", _P_I32),
                ("tag", _P_I32), ("active", _P_I32), ("transform_type", _P_I32), ("position", _P_F64),
                ("basis", _P_F64), ("velocity", _P_F64), ("quaternion", _P_F64), ("omega", _P_F64),
                ("force", _P_F64), ("torque", _P_F64), ("memory", ContactMemory)]


def read_reload_particles(lib, path, binary=False):
    """Parses a particle file of a reload (text or hybrid binary) with
    grains_gpu_reload_open / _get: a dict of per-particle arrays (file order)
    and 'memory' with every contact-map entry (owner = holder id)."""
    h = C.c_void_p()
    rc = lib.fn["reload_open"](os.fsencode(path), 1 if binary else 0, C.byref(h))
    try:
        if rc:
            buf = C.create_string_buffer(4096)
            if h:
                lib.fn["reload_last_error"](h, buf, 4096)
            raise error_for(rc, buf.value.decode(errors="replace"))
        d = ReloadData()
        lib.fn["reload_get"](h, C.byref(d))
        n, m = d.n_particles, d.n_memory
        out = {k: np.zeros(n, np.int32) for k in ["geom_type", "id", "tag", "active", "transform_type"]}
        for k, w in [("position", 3), ("basis", 9), ("velocity", 3), ("quaternion", 4), ("omega", 3),
                     ("force", 3), ("torque", 3)]:
            out[k] = np.zeros((n, w))
        mem = {"owner": np.zeros(m, np.int32), "other": np.zeros(m, np.int32), "kdelta": np.zeros((m, 3)),
               "prev_normal": np.zeros((m, 3)), "spring_torque": np.zeros((m, 3))}
        for k in ["geom_type", "id", "tag", "active", "transform_type"]:
            setattr(d, k, _ptr(out[k], C.c_int32))
        for k in ["position", "basis", "velocity", "quaternion", "omega", "force", "torque"]:
            setattr(d, k, _ptr(out[k], C.c_double))
        d.memory.n = m
        d.memory.owner, d.memory.other = _ptr(mem["owner"], C.c_int32), _ptr(mem["other"], C.c_int32)
        d.memory.kdelta = _ptr(mem["kdelta"], C.c_double)
        d.memory.prev_normal = _ptr(mem["prev_normal"], C.c_double)
        d.memory.spring_torque = _ptr(mem["spring_torque"], C.c_double)
        rc = lib.fn["reload_get"](h, C.byref(d))
        if rc:
            raise error_for(rc, "reload_get failed")
        out["memory"] = mem
        return out
    finally:
        if h:
            lib.fn["reload_close"](h)


def format_double(lib, x, digits):
    """GrainsExec::doubleToString(ios::scientific, digits, x) with the library's formatter (host)."""
    buf = C.create_string_buffer(64)
    n = C.c_int32()
    rc = lib.fn["format_double"](float(x), digits, buf, 64, C.byref(n))
    if rc:
        raise error_for(rc, "format_double failed")
    return buf.value.decode()


def format_doubles_on_device(lib, values, digits):
    """The same formatter run on the device over an array: one value per line."""
    x = np.ascontiguousarray(values, dtype=np.float64)
    cap = 32 * len(x) + 64
    buf = C.create_string_buffer(cap)
    n = C.c_int64()
    rc = lib.fn["format_doubles"](_ptr(x, C.c_double), len(x), digits, buf, cap, C.byref(n))
    if rc:
        raise error_for(rc, "format_doubles failed")
    return buf.raw[:n.value].decode()


class GrainsLib:
    """A loaded implementation of the grains_gpu C ABI (entry points `prefix + name`)."""

    def __init__(self, path, prefix="grains_gpu_"):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.prefix = prefix
        self.dll = C.CDLL(path)
        self.fn = {}
        for name, args in list(_SIGS.items()) + list(_GPU_ONLY.items()):
            sym = prefix + name
            if not hasattr(self.dll, sym):
                if name in _GPU_ONLY or name in _OPTIONAL:
                    continue
                raise AttributeError("%s does not export %s" % (path, sym))
            f = getattr(self.dll, sym)
            f.argtypes = args
            f.restype = C.c_int
            self.fn[name] = f
        if "set_gjk_tolerance" not in self.fn and hasattr(self.dll, prefix + "set_gjk_tolerance"):
            f = getattr(self.dll, prefix + "set_gjk_tolerance")
            f.argtypes = [_VP, C.c_double]
            f.restype = C.c_int
            self.fn["set_gjk_tolerance"] = f
        if hasattr(self.dll, prefix + "set_polyhedron_support"):  # oracle-only test switch
            f = getattr(self.dll, prefix + "set_polyhedron_support")
            f.argtypes = [_VP, C.c_int32]
            f.restype = C.c_int
            self.fn["set_polyhedron_support"] = f

    def shape_properties(self, shape_type, params):
        p = np.ascontiguousarray(params, dtype=np.float64)
        vol, circ = C.c_double(), C.c_double()
        inertia = (C.c_double * 3)()
        rc = self.fn["shape_properties"](shape_type, p.ctypes.data_as(_P_F64), len(p), C.byref(vol),
                                         C.byref(circ), inertia)
        if rc:
            raise GrainsError(rc, "shape_properties failed")
        return vol.value, circ.value, np.array(inertia[:])


def _ptr(a, ctype):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if n is None else a.reshape(-1)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Simulation:
    """One context of the DEM step (a drop-in for the LinkedCell App + integrator)."""

    def __init__(self, lib, precision=MIXED, max_particles=1024, n_systems=1, history_capacity=0, device=0,
                 max_materials=4, max_obstacles=0):
        self.lib = lib
        cfg = Config()
        cfg.precision = precision
        cfg.device = device
        cfg.n_systems = n_systems
        cfg.history_capacity = history_capacity
        cfg.max_particles = max_particles
        cfg.max_obstacles = max_obstacles
        cfg.max_materials = max_materials
        self.ctx = _VP()
        rc = lib.fn["create"](C.byref(cfg), C.byref(self.ctx))
        if rc:
            msg = self.last_error() if self.ctx else "create failed"
            if self.ctx:
                lib.fn["destroy"](self.ctx)
                self.ctx = _VP()
            raise error_for(rc, msg)
        self.n = 0
        self.n_systems = n_systems
        self._keep = []

    def close(self):
        if self.ctx:
            self.lib.fn["destroy"](self.ctx)
            self.ctx = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def last_error(self):
        buf = C.create_string_buffer(4096)
        self.lib.fn["last_error"](self.ctx, buf, 4096)
        return buf.value.decode(errors="replace")

    def _check(self, rc):
        if rc:
            raise error_for(rc, self.last_error())

    # ---- set-up ----
    def set_domain(self, system, origin, size, cell_size, gravity=(0.0, 0.0, -9.81)):
        d = Domain()
        d.origin[:] = list(origin)
        d.size[:] = list(size)
        d.cell_size = cell_size
        d.gravity[:] = list(gravity)
        self._check(self.lib.fn["set_domain"](self.ctx, system, C.byref(d)))

    def add_shape(self, shape_type, params):
        p = f64(params)
        sid = C.c_int32()
        self._check(self.lib.fn["add_shape"](self.ctx, shape_type, _ptr(p, C.c_double), len(p), C.byref(sid)))
        return sid.value

    def set_contact_law(self, system, mat_a, mat_b, law, params):
        p = f64(params)
        self._check(self.lib.fn["set_contact_law"](self.ctx, system, mat_a, mat_b, law, _ptr(p, C.c_double), len(p)))

    def set_obstacles(self, system, obstacles):
        arr = (Obstacle * max(1, len(obstacles)))()
        for k, o in enumerate(obstacles):
            ob = arr[k]
            ob.id = o["id"]
            ob.shape = o["shape"]
            ob.material = o.get("material", 0)
            ob.moving = int(o.get("moving", 0))
            ob.crust = o["crust"]
            ob.transform[:] = [float(x) for x in o["transform"]]
            ob.velocity[:] = list(o.get("velocity", (0.0, 0.0, 0.0)))
            ob.omega[:] = list(o.get("omega", (0.0, 0.0, 0.0)))
            ob.rotation_center[:] = list(o.get("rotation_center", (0.0, 0.0, 0.0)))
        self._check(self.lib.fn["set_obstacles"](self.ctx, system, len(obstacles), arr))

    def set_collision_algorithm(self, algorithm):
        """GJK (0, Johnson's) or GJK_SV (1, signed volumes) for non-spherical pairs."""
        self._check(self.lib.fn["set_collision_algorithm"](self.ctx, algorithm))

    def set_collision_options(self, tolerance=1e-10, acceleration=False, history=False):
        """The Tolerance, Acceleration and History attributes of the
        reference's <CollisionDetection> element: the GJK optimality-gap
        tolerance, Nesterov-accelerated search directions, and the warm start
        of each convex pair from its last GJK iterate."""
        self._check(self.lib.fn["set_collision_options"](self.ctx, float(tolerance), int(bool(acceleration)),
                                                          int(bool(history))))

    def set_obstacle_loadings(self, system, loadings):
        """Imposed obstacle motions: dicts with obstacle_id, type, t_start,
        t_end and the type's fields (vector, center, amplitude, period,
        phase_deg as 3-sequences or scalars)."""
        arr = (ObstacleLoading * max(1, len(loadings)))()

        def three(v):
            v = np.atleast_1d(np.asarray(v, dtype=float))
            return list(v) + [0.0] * (3 - len(v))
        for k, l in enumerate(loadings):
            g = arr[k]
            g.obstacle_id = l["obstacle_id"]
            g.type = l["type"]
            g.t_start = l.get("t_start", 0.0)
            g.t_end = l.get("t_end", 1.0e9)
            g.vector[:] = three(l.get("vector", 0.0))
            g.center[:] = three(l.get("center", 0.0))
            g.has_center = 1 if "center" in l else 0
            g.amplitude[:] = three(l.get("amplitude", 0.0))
            g.period[:] = three(l.get("period", 0.0))
            g.phase_deg[:] = three(l.get("phase_deg", 0.0))
        self._check(self.lib.fn["set_obstacle_loadings"](self.ctx, system, len(loadings), arr))

    # ---- state ----
    def upload(self, p):
        n = len(p["id"])
        arrs = {
            "id": i32(p["id"]),
            "system": i32(p["system"]) if p.get("system") is not None else None,
            "shape": i32(p["shape"]),
            "material": i32(p["material"]),
            "radius": f64(p["radius"]),
            "crust": f64(p["crust"]),
            "mass": f64(p["mass"]),
            "inertia": f64(p["inertia"]),
            "position": f64(p["position"]),
            "quaternion": f64(p["quaternion"]),
            "basis": f64(p["basis"]) if p.get("basis") is not None else None,
            "velocity": f64(p["velocity"]),
            "omega": f64(p["omega"]),
            "force": f64(p["force"]) if p.get("force") is not None else None,
            "torque": f64(p["torque"]) if p.get("torque") is not None else None,
        }
        s = Particles()
        s.n = n
        for k, a in arrs.items():
            setattr(s, k, _ptr(a, C.c_int32 if a is not None and a.dtype == np.int32 else C.c_double))
        self._keep = list(arrs.values())
        self._check(self.lib.fn["upload_particles"](self.ctx, C.byref(s)))
        self.n = n

    def update(self, p):
        """Overwrites position, quaternion, (basis), velocity and omega of the
        uploaded particles (upload order) keeping contact memory and forces."""
        arrs = {k: f64(p[k]) for k in ["position", "quaternion", "velocity", "omega"]}
        arrs["basis"] = f64(p["basis"]) if p.get("basis") is not None else None
        s = Particles()
        s.n = self.n
        for k, a in arrs.items():
            setattr(s, k, _ptr(a, C.c_double))
        self._keep_update = list(arrs.values())
        self._check(self.lib.fn["update_particles"](self.ctx, C.byref(s)))

    def set_fluid(self, fluid_density, corrected=True, particle_density=None):
        """Immersed particles (the fluid set-up of GrainsCoupledWithFluid):
        buoyant weights m (1 - rho_f / rho_p) g and, when `corrected`,
        accelerations divided by 1 - rho_f / rho_p.  particle_density: rho_p
        per particle in upload order."""
        d = f64(particle_density) if particle_density is not None else None
        self._keep_fluid = d
        self._check(self.lib.fn["set_fluid"](self.ctx, float(fluid_density), int(bool(corrected)),
                                             _ptr(d, C.c_double) if d is not None else None))

    def set_hydro_forces(self, force=None, torque=None):
        """The fluid's force and torque on every particle (upload order, 3
        each), added to every force evaluation; None removes them."""
        f = f64(force) if force is not None else None
        t = f64(torque) if torque is not None else None
        self._keep_hydro = (f, t)
        self._check(self.lib.fn["set_hydro_forces"](self.ctx, _ptr(f, C.c_double) if f is not None else None,
                                                    _ptr(t, C.c_double) if t is not None else None))

    def set_velocities(self, velocity, omega):
        """Translational and angular (world) velocities of every particle,
        upload order."""
        v, w = f64(velocity), f64(omega)
        self._check(self.lib.fn["set_velocities"](self.ctx, _ptr(v, C.c_double), _ptr(w, C.c_double)))

    def fluid_step(self, dt_fluid, min_dt, max_dt, ndt, time):
        """The DEM steps of one fluid step (GrainsCoupledWithFluid::
        Simulation): returns (the new step count, the new time)."""
        n = C.c_int64(int(ndt))
        t = C.c_double(float(time))
        self._check(self.lib.fn["fluid_step"](self.ctx, float(dt_fluid), float(min_dt), float(max_dt), C.byref(n),
                                              C.byref(t)))
        return n.value, t.value

    def fluid_features(self):
        """The rigid bodies for the fluid solver (GrainsToFluid, tokenised as
        GrainsToBasilisk passes it on), as a str."""
        n = C.c_int64(0)
        self._check(self.lib.fn["fluid_features"](self.ctx, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        self._check(self.lib.fn["fluid_features"](self.ctx, buf, n.value, C.byref(n)))
        return buf.value.decode()

    def update_rows(self, rows, p):
        """Overwrites the kinematic state of the particles at upload indices
        `rows` (distinct) with the arrays of `p` (one entry per row: position,
        quaternion, velocity, omega, and basis when given); the other
        particles are untouched."""
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        arrs = {k: f64(p[k]) for k in ["position", "quaternion", "velocity", "omega"]}
        arrs["basis"] = f64(p["basis"]) if p.get("basis") is not None else None
        s = Particles()
        s.n = len(rows)
        for k, a in arrs.items():
            setattr(s, k, _ptr(a, C.c_double))
        self._keep_update = list(arrs.values()) + [rows]
        self._check(self.lib.fn["update_particle_rows"](self.ctx, len(rows), rows.ctypes.data_as(C.POINTER(C.c_int64)),
                                                        C.byref(s)))

    def download(self, out=None):
        """The state in upload order.  `out`: preallocated arrays to fill (for
        example views of pinned host memory), keyed like the result; fields
        left out of it are not downloaded."""
        n = self.n
        if out is None:
            out = {
                "id": np.zeros(n, np.int32),
                "position": np.zeros((n, 3)),
                "quaternion": np.zeros((n, 4)),
                "basis": np.zeros((n, 9)),
                "velocity": np.zeros((n, 3)),
                "omega": np.zeros((n, 3)),
                "force": np.zeros((n, 3)),
                "torque": np.zeros((n, 3)),
                "coordination": np.zeros(n, np.int32),
            }
        for k, a in out.items():
            assert a.flags["C_CONTIGUOUS"] and a.dtype == (np.int32 if k in ("id", "coordination") else np.float64)
        s = Particles()
        s.n = n
        for k, a in out.items():
            setattr(s, k, _ptr(a, C.c_int32 if a.dtype == np.int32 else C.c_double))
        self._check(self.lib.fn["download_particles"](self.ctx, C.byref(s)))
        return out

    def upload_contact_memory(self, mem):
        n = len(mem["owner"])
        owner, other = i32(mem["owner"]), i32(mem["other"])
        kd, pn, sp = f64(mem["kdelta"]), f64(mem["prev_normal"]), f64(mem["spring_torque"])
        m = ContactMemory()
        m.n = n
        m.owner, m.other = _ptr(owner, C.c_int32), _ptr(other, C.c_int32)
        m.kdelta, m.prev_normal, m.spring_torque = _ptr(kd, C.c_double), _ptr(pn, C.c_double), _ptr(sp, C.c_double)
        sy = i32(mem["system"]) if mem.get("system") is not None else None
        m.system = _ptr(sy, C.c_int32) if sy is not None else None
        self._check(self.lib.fn["upload_contact_memory"](self.ctx, C.byref(m)))

    def contact_memory(self, cap=None):
        cap = cap or max(64, 32 * self.n)
        owner, other, sy = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        kd, pn, sp = np.zeros((cap, 3)), np.zeros((cap, 3)), np.zeros((cap, 3))
        m = ContactMemory()
        m.n = cap
        m.owner, m.other = _ptr(owner, C.c_int32), _ptr(other, C.c_int32)
        m.kdelta, m.prev_normal, m.spring_torque = _ptr(kd, C.c_double), _ptr(pn, C.c_double), _ptr(sp, C.c_double)
        m.system = _ptr(sy, C.c_int32)
        self._check(self.lib.fn["download_contact_memory"](self.ctx, C.byref(m)))
        k = m.n
        return {"owner": owner[:k], "other": other[:k], "kdelta": kd[:k], "prev_normal": pn[:k],
                "spring_torque": sp[:k], "system": sy[:k]}

    def obstacles(self, system, n):
        """Poses of the first n obstacles of `system` after their imposed
        motion: (n, 12) = row-major rotation matrix, then the centre."""
        out = np.zeros((n, 12))
        self._check(self.lib.fn["download_obstacles"](self.ctx, system, n, _ptr(out, C.c_double)))
        return out

    # ---- the step ----
    def compute_forces(self, time, dt):
        self._check(self.lib.fn["compute_forces"](self.ctx, time, dt))

    def move(self, time, dt_vel, dt_disp):
        self._check(self.lib.fn["move"](self.ctx, time, dt_vel, dt_disp))

    def link_update(self, time=0.0, dt=0.0):
        self._check(self.lib.fn["link_update"](self.ctx, time, dt))

    def advance_velocity(self, time, dt_vel):
        self._check(self.lib.fn["advance_velocity"](self.ctx, time, dt_vel))

    def initialize_leapfrog(self, time, dt):
        self._check(self.lib.fn["initialize_leapfrog"](self.ctx, time, dt))

    def step(self, n_steps, time, dt):
        t = C.c_double(time)
        self._check(self.lib.fn["step"](self.ctx, n_steps, C.byref(t), dt))
        return t.value

    def synchronize(self):
        if "synchronize" in self.lib.fn:
            self._check(self.lib.fn["synchronize"](self.ctx))

    # ---- diagnostics ----
    def candidate_pairs(self, system=0, include_obstacles=False, cap=None):
        cap = cap or max(1024, 40 * self.n)
        buf = np.zeros(2 * cap, np.int32)
        n = C.c_int64()
        self._check(self.lib.fn["get_candidate_pairs"](self.ctx, system, int(include_obstacles), cap,
                                                       _ptr(buf, C.c_int32), C.byref(n)))
        return buf[: 2 * n.value].reshape(-1, 2)

    def contact_pairs(self, system=0, cap=None):
        cap = cap or max(1024, 16 * self.n)
        buf = np.zeros(2 * cap, np.int32)
        n = C.c_int64()
        self._check(self.lib.fn["get_contact_pairs"](self.ctx, system, cap, _ptr(buf, C.c_int32), C.byref(n)))
        return buf[: 2 * n.value].reshape(-1, 2)

    def contact_forces(self, system=0, cap=None):
        """(pairs (k, 2), force on the lower id (k, 3)) of the last compute_forces."""
        cap = cap or max(1024, 16 * self.n)
        buf = np.zeros(2 * cap, np.int32)
        f = np.zeros(3 * cap, np.float64)
        n = C.c_int64()
        self._check(self.lib.fn["get_contact_forces"](self.ctx, system, cap, _ptr(buf, C.c_int32),
                                                      _ptr(f, C.c_double), C.byref(n)))
        return buf[: 2 * n.value].reshape(-1, 2), f[: 3 * n.value].reshape(-1, 3)

    # ---- reload and RawData files ----
    def set_record_attributes(self, geom_type=None, tag=None, active=None, transform_type=None):
        """Reload-file attributes per particle (upload order); None keeps them."""
        arrs = [None if a is None else i32(a) for a in (geom_type, tag, active, transform_type)]
        ptrs = [_ptr(a, C.c_int32) for a in arrs]
        self._check(self.lib.fn["set_record_attributes"](self.ctx, self.n, *ptrs))

    def write_reload_particles(self, path, binary=False):
        """The particle file of a reload (text, or hybrid binary); returns its size."""
        nb = C.c_int64()
        self._check(self.lib.fn["write_reload_particles"](self.ctx, os.fsencode(path), 1 if binary else 0,
                                                          C.byref(nb)))
        return nb.value

    def write_rawdata(self, root, time, n_total=None, binary=False, truncate=False, system=0):
        """One RawData output time (the ten time-series files and the type file)."""
        nb = C.c_int64()
        n_total = self.n if n_total is None else n_total
        self._check(self.lib.fn["write_rawdata"](self.ctx, os.fsencode(root), float(time), system, n_total,
                                                 1 if binary else 0, 1 if truncate else 0, C.byref(nb)))
        return nb.value

    def stats(self):
        st = Stats()
        self._check(self.lib.fn["get_stats"](self.ctx, C.byref(st)))
        return {f: getattr(st, f) for f, _ in Stats._fields_ if f != "reserved"}

    def reset_stats(self):
        self._check(self.lib.fn["reset_stats"](self.ctx))

    def set_gjk_tolerance(self, tol):
        self._check(self.lib.fn["set_gjk_tolerance"](self.ctx, tol))

    def set_polyhedron_support(self, mode):
        """Oracle only: 0 the reference's polyhedron support (a hill climb from
        the vertex each body kept), 1 the order-independent arg-max, 2 the
        CUDA path's hill climb that every GJK run starts at vertex 0."""
        self._check(self.lib.fn["set_polyhedron_support"](self.ctx, int(mode)))

    # ---- tuning (CUDA implementation only) ----
    def tuning(self):
        t = Tuning()
        self._check(self.lib.fn["get_tuning"](self.ctx, C.byref(t)))
        return {"cell_factor": t.cell_factor, "contacts_block": t.contacts_block, "forces_block": t.forces_block,
                "list_capacity": t.list_capacity, "gather_every": t.gather_every, "persistent": t.persistent}

    def set_tuning(self, cell_factor=1.0, contacts_block=256, forces_block=128, list_capacity=0, gather_every=16,
                   persistent=0):
        t = Tuning(cell_factor, contacts_block, forces_block, list_capacity, gather_every, persistent)
        self._check(self.lib.fn["set_tuning"](self.ctx, C.byref(t)))

    def autotune(self, time, dt, trial_steps=100):
        """Picks and applies the fastest tuning; returns (tuning dict, ms of trial_steps)."""
        t, ms = Tuning(), C.c_double()
        self._check(self.lib.fn["autotune"](self.ctx, time, dt, trial_steps, C.byref(t), C.byref(ms)))
        return ({"cell_factor": t.cell_factor, "contacts_block": t.contacts_block, "forces_block": t.forces_block,
                 "list_capacity": t.list_capacity, "gather_every": t.gather_every, "persistent": t.persistent},
                ms.value)

    # ---- benchmark helpers (CUDA implementation only) ----
    def stream_handle(self):
        h = _VP()
        self._check(self.lib.fn["get_stream"](self.ctx, C.byref(h)))
        return h.value

    def set_barrier_test(self, polls=1 << 24, skip_block=-1):
        """Test hook of the persistent launch's bounded grid-barrier wait."""
        self._check(self.lib.fn["set_barrier_test"](self.ctx, polls, skip_block))

    def launches_per_step(self):
        n = C.c_int64()
        self._check(self.lib.fn["launches_per_step"](self.ctx, C.byref(n)))
        return n.value

    def profile_kernels(self, n_steps, time, dt, max_kernels=8):
        t = C.c_double(time)
        names = C.create_string_buffer(1024)
        ms = (C.c_double * max_kernels)()
        launches = (C.c_int64 * max_kernels)()
        nk = C.c_int32()
        self._check(self.lib.fn["profile_kernels"](self.ctx, n_steps, C.byref(t), dt, names, 1024, ms, launches,
                                                   max_kernels, C.byref(nk)))
        keys = names.value.decode().split("\n")
        return t.value, {keys[i]: (ms[i], launches[i]) for i in range(nk.value)}


class Adjoint:
    """Differentiable run of a Simulation's current state (spheres, static box
    walls) and its adjoint: grains_gpu_adjoint_* of the C ABI."""

    def __init__(self, sim, checkpoint_every=100):
        self.sim = sim
        self.h = _VP()
        rc = sim.lib.fn["adjoint_create"](sim.ctx, checkpoint_every, C.byref(self.h))
        if rc:
            msg = self.last_error() if self.h else "adjoint_create failed"
            self.close()
            raise error_for(rc, msg)
        n = C.c_int32()
        self._check(sim.lib.fn["adjoint_law_slots"](self.h, C.byref(n)))
        self.n_law_slots = n.value

    def close(self):
        if self.h:
            self.sim.lib.fn["adjoint_destroy"](self.h)
            self.h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self):
        buf = C.create_string_buffer(4096)
        self.sim.lib.fn["adjoint_last_error"](self.h, buf, 4096)
        return buf.value.decode(errors="replace")

    def _check(self, rc):
        if rc:
            raise error_for(rc, self.last_error())

    def forward(self, n_steps, dt):
        """Final state {position, velocity, omega} (n, 3) in upload order."""
        n = self.sim.n
        x, v, w = (np.zeros(3 * n) for _ in range(3))
        self._check(self.sim.lib.fn["adjoint_forward"](self.h, n_steps, dt, _ptr(x, C.c_double), _ptr(v, C.c_double),
                                                       _ptr(w, C.c_double)))
        return {"position": x.reshape(n, 3), "velocity": v.reshape(n, 3), "omega": w.reshape(n, 3)}

    def signature(self):
        """(hash of the contact sets of the last forward run, total contacts)."""
        sig, cnt = C.c_uint64(), C.c_int64()
        self._check(self.sim.lib.fn["adjoint_contact_signature"](self.h, C.byref(sig), C.byref(cnt)))
        return sig.value, cnt.value

    def backward(self, dposition=None, dvelocity=None, domega=None):
        """Gradients of the loss w.r.t. the initial state and, in 'laws', an
        (n_law_slots, 4) array of dL/d(kn, en, muc, kt) per law-table slot."""
        n = self.sim.n

        def arg(a):
            return None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        gx, gv, gw = arg(dposition), arg(dvelocity), arg(domega)
        ox, ov, ow = (np.zeros(3 * n) for _ in range(3))
        gl = np.zeros(4 * self.n_law_slots)
        self._check(self.sim.lib.fn["adjoint_backward"](self.h, _ptr(gx, C.c_double), _ptr(gv, C.c_double),
                                                        _ptr(gw, C.c_double), _ptr(ox, C.c_double),
                                                        _ptr(ov, C.c_double), _ptr(ow, C.c_double),
                                                        _ptr(gl, C.c_double), len(gl)))
        return {"position": ox.reshape(n, 3), "velocity": ov.reshape(n, 3), "omega": ow.reshape(n, 3),
                "laws": gl.reshape(-1, 4)}
