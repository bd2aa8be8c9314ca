"""Shared helpers of the parity tests: run the same scenario through the CUDA
library and the CPU oracle and compare."""
import os

import numpy as np

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED, Simulation


def make(lib, sc, precision=FP64, history_capacity=0):
    sim = Simulation(lib, precision, max_particles=max(sc.n, 1), n_systems=len(sc.domains),
                     history_capacity=history_capacity)
    S.apply(sim, sc)
    return sim


def pair_set(a):
    return set(map(tuple, np.asarray(a).reshape(-1, 2).tolist()))


def rel_err(a, b, floor):
    """max |a - b| / max(|b|, floor) over rows (vector norms)."""
    a, b = np.asarray(a), np.asarray(b)
    num = np.linalg.norm(a - b, axis=-1)
    den = np.maximum(np.linalg.norm(b, axis=-1), floor)
    return float(np.max(num / den)) if len(num) else 0.0


def perturbed_cluster(n=200, seed=0, sigma=0.2, spacing=2.04):
    """A cluster of spheres with velocities large enough to collide in a few
    steps and with walls in reach."""
    return S.small_box(n, seed=seed, velocity_sigma=sigma, spacing=spacing)


def rel_err_quantile(a, b, floor, q):
    """q-quantile over rows of |a - b| / max(|b|, floor)."""
    a, b = np.asarray(a), np.asarray(b)
    num = np.linalg.norm(a - b, axis=-1)
    den = np.maximum(np.linalg.norm(b, axis=-1), floor)
    return float(np.quantile(num / den, q)) if len(num) else 0.0


def check_contact_forces(fg, fo, floor, precision):
    """Per-contact forces: FP64 at rounding level; mixed precision within
    1e-5 for every contact (the north star's bar).  The mixed law forms its
    normal part (the elastic and viscous terms, which nearly cancel on a
    contact about to open) in double, so FP32 rounding enters only the
    tangential part and the final force, about 1e-7 of the force."""
    if precision == FP64:
        assert rel_err(fg, fo, floor) < 1e-12
    else:
        assert rel_err(fg, fo, floor) < 1e-5


TANGENT_SO = None


def tangent_run(sc, n_steps, dir_v0=None, dir_laws=None, n_mat=4):
    """The oracle's forward-mode run (oracle/tangent_oracle.cpp) of scenario
    `sc` (spheres, one system, box walls): final state and, for each
    direction, the derivative of the final state along (dir_v0[d] (n, 3),
    dir_laws[d] (n_mat^2, 4) = d(kn, en, muc, kt) per law slot)."""
    import ctypes as C
    import os
    from pacific_b200 import scenarios as S
    global TANGENT_SO
    if TANGENT_SO is None:
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        TANGENT_SO = C.CDLL(os.path.join(root, "oracle", "_build", "libgrains_tangent.so"))
    p = sc.particles
    n = len(p["id"])
    d = sc.domains[0]
    dom = np.concatenate([np.asarray(d["origin"], float), np.asarray(d["size"], float), [d["cell_size"]],
                          np.asarray(d["gravity"], float)])
    walls = []
    for o in sc.obstacles[0]:
        t, prm = sc.shapes[o["shape"]]
        assert t == S.BOX
        e = np.abs(np.asarray(prm, float)) / 2.0
        vol = 8.0 * e[0] * e[1] * e[2]
        walls.append(list(o["transform"]) + list(e) + [o["crust"], o["material"], (0.75 / np.pi * vol) ** (1.0 / 3.0)])
    laws = np.zeros((n_mat * n_mat, 10))
    laws[:, 0] = -1
    for a, b, law, prm in sc.laws[0]:
        if law == S.HOOKE_MEMORY:
            row = [1, prm[0], prm[1], prm[2], prm[3], prm[4], prm[5], prm[6], prm[7], 0.0]
        else:
            row = [0, prm[0], prm[1], prm[2], prm[3], 0.0, 0.0, 0.0, 0.0, prm[4]]
        laws[a * n_mat + b] = row
        laws[b * n_mat + a] = row
    nd = 0 if dir_v0 is None else len(dir_v0)

    def f64(a):
        return np.ascontiguousarray(a, dtype=np.float64)
    x0, v0, w0 = f64(p["position"]), f64(p["velocity"]), f64(p["omega"])
    rad, mass, inertia, crust = f64(p["radius"]), f64(p["mass"]), f64(np.asarray(p["inertia"])[:, 0]), f64(p["crust"])
    mat = np.ascontiguousarray(p["material"], dtype=np.int32)
    wl = f64(np.asarray(walls).reshape(-1))
    dv = f64(np.zeros((max(nd, 1), n, 3)) if dir_v0 is None else dir_v0)
    dl = f64(np.zeros((max(nd, 1), n_mat * n_mat, 4)) if dir_laws is None else dir_laws)
    x, v, w = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n)
    tx, tv, tw = (np.zeros(max(nd, 1) * 3 * n) for _ in range(3))
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    fn = TANGENT_SO.grains_tangent_run
    fn.restype = C.c_int
    rc = fn(C.c_int(n), P(x0), P(v0), P(w0), P(rad), P(mass), P(inertia), P(crust),
            mat.ctypes.data_as(C.POINTER(C.c_int)), P(f64(dom)), C.c_int(len(walls)), P(wl), C.c_int(n_mat),
            P(f64(laws)), C.c_int(n_steps), C.c_double(sc.dt), C.c_int(nd), P(dv), P(dl), P(x), P(v), P(w),
            P(tx), P(tv), P(tw))
    assert rc == 0, "tangent run failed (contact or motion error)"
    fin = {"position": x.reshape(n, 3), "velocity": v.reshape(n, 3), "omega": w.reshape(n, 3)}
    tan = {"position": tx.reshape(-1, n, 3)[:nd], "velocity": tv.reshape(-1, n, 3)[:nd],
           "omega": tw.reshape(-1, n, 3)[:nd]}
    return fin, tan


# ---- reload / RawData fixtures (tests/golden/io_*.npz) ----
RAW_FILES = ["_position_x.dat", "_position_y.dat", "_position_z.dat", "_translational_velocity_x.dat",
             "_translational_velocity_y.dat", "_translational_velocity_z.dat", "_angular_velocity_x.dat",
             "_angular_velocity_y.dat", "_angular_velocity_z.dat", "_coordinationNumber.dat", "_particleType.dat"]


def read_fixture_reload(reader_lib, z, tmpdir, binary=False):
    """The reference's particle file of fixture z, parsed by the library's reader."""
    from pacific_b200.abi import read_reload_particles
    path = os.path.join(str(tmpdir), "ref_reload" + (".bin" if binary else ".txt"))
    with open(path, "wb") as f:
        f.write(bytes(z["reload_bin" if binary else "reload_text"]))
    return read_reload_particles(reader_lib, path, binary)


def fixture_scenario(z, r):
    """The fixture's scenario with the particles of the parsed file r (file
    order) and the static data the fixture recorded for them."""
    import json
    spec = json.loads(str(z["spec"]))
    doms = [dict(origin=np.array(d["origin"]), size=np.array(d["size"]), cell_size=d["cell_size"],
                 gravity=tuple(d["gravity"])) for d in spec["domains"]]
    laws = [[(l[0], l[1], l[2], l[3]) for l in ls] for ls in spec["laws"]]
    p = dict(id=r["id"], system=None, shape=z["static_shape"], material=z["static_material"],
             radius=z["static_radius"], crust=z["static_crust"], mass=z["static_mass"], inertia=z["static_inertia"],
             position=r["position"], quaternion=r["quaternion"], basis=r["basis"], velocity=r["velocity"],
             omega=r["omega"], force=r["force"], torque=r["torque"])
    return S.Scenario(spec["name"], [tuple(s) for s in spec["shapes"]], doms, laws, spec["obstacles"], p,
                      spec["dt"], spec["n_steps"])


def load_fixture_state(lib, z, r, precision=FP64):
    """A context holding exactly the state the reference wrote: particles,
    torsors, bases, both sides of every contact memory and the record
    attributes."""
    sc = fixture_scenario(z, r)
    sim = make(lib, sc, precision)
    sim.upload_contact_memory(r["memory"])
    sim.set_record_attributes(r["geom_type"], r["tag"], r["active"], r["transform_type"])
    return sc, sim
