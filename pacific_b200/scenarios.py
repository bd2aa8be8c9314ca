"""Seeded synthetic inputs of the benchmark workloads (no public dataset exists
for the Grains3D DEM step; these stand in for the reference's insertion).

Every generator returns a `Scenario`: shapes, per-system domains, contact laws,
wall obstacles and particle arrays, ready for `apply(sim, scenario)` on any
implementation of the grains_gpu C ABI.  Masses and inertias follow the
reference's formulas (Particle.cpp:158-163, Sphere.cpp:61-70,152-155,
Box.cpp:181-210, Cylinder.cpp:61-100).  Walls are thin Box obstacles whose
inner faces lie on the domain faces, like the reference's test layouts
(Tests/data/spheres-settling-new-grains/Grains/Init/insert.xml).
"""
import math
from dataclasses import dataclass, field

import numpy as np

from .abi import BOX, CYLINDER, HERTZ, HERTZ_MEMORY, HOOKE_MEMORY, POLYHEDRON, SPHERE  # noqa: F401

MM = 1.0e-3
PI = 3.14159265358979323846


@dataclass
class Scenario:
    name: str
    shapes: list                     # [(type, params)]
    domains: list                    # per system: dict(origin, size, cell_size, gravity)
    laws: list                       # per system: [(mat_a, mat_b, law, params)]
    obstacles: list                  # per system: [dict(id, shape_index, material, crust, transform, ...)]
    particles: dict                  # numpy arrays; 'shape' holds shape-list indices
    dt: float
    n_steps: int
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.particles["id"])


def sphere_mass_inertia(r, rho):
    """mass = rho * 4 pi r^3 / 3 and principal inertia rho * 8 pi r^5 / 15."""
    r = np.asarray(r, dtype=np.float64)
    vol = np.array([4.0 * PI * math.pow(x, 3.0) / 3.0 for x in r.ravel()]).reshape(r.shape)
    i0 = np.array([8.0 * PI * math.pow(x, 5.0) / 15.0 for x in r.ravel()]).reshape(r.shape)
    return rho * vol, np.repeat((i0 * rho)[:, None], 3, axis=1)


def hooke_memory_params(kn, en, muc, kt, etat=-1.0, mur=0.0, etarpf=0.0, epst=0.0):
    """HookeMemory parameters in C ABI order.  epst = 0 is the effective value
    when the XML omits it (the fallback writes key "eps" but the model reads
    "epst", HookeMemoryContactForceModel.cpp:21, 300-306)."""
    return [kn, en, etat, muc, kt, mur, etarpf, epst]


def box_walls(lo, hi, faces, thickness, crust, shape_offset, id_start, material=1):
    """Thin box walls on the chosen faces of the box [lo, hi].

    faces: subset of 'xX yY zZ' letters (lower case = lower face).  Returns
    (shapes, obstacles); obstacle 'shape' indexes into the returned shapes
    list shifted by shape_offset.
    """
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    size = hi - lo
    t = thickness
    shapes, obs = [], []
    for k, f in enumerate(faces):
        axis = "xyz".index(f.lower())
        upper = f.isupper()
        edges = size + 2 * t
        edges[axis] = t
        centre = (lo + hi) / 2.0
        centre[axis] = (hi[axis] + t / 2.0) if upper else (lo[axis] - t / 2.0)
        shapes.append((BOX, list(edges)))
        obs.append(dict(id=id_start - k, shape=shape_offset + len(shapes) - 1, material=material, crust=crust,
                        transform=[1, 0, 0, 0, 1, 0, 0, 0, 1, *centre]))
    return shapes, obs


def lattice(n, lo, hi, spacing, margin, jitter, rng):
    """First n sites of a cubic lattice inside [lo, hi] (x fastest, then y, z),
    with a uniform jitter in [-jitter, jitter] per coordinate."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    counts = [int(math.floor((hi[a] - lo[a] - 2 * margin) / spacing + 1e-9)) + 1 for a in range(3)]
    per_layer = counts[0] * counts[1]
    if per_layer * counts[2] < n:
        raise ValueError("lattice holds %d sites < %d" % (per_layer * counts[2], n))
    k = np.arange(n)
    ix, iy, iz = k % counts[0], (k // counts[0]) % counts[1], k // per_layer
    pos = np.stack([lo[0] + margin + ix * spacing, lo[1] + margin + iy * spacing, lo[2] + margin + iz * spacing], 1)
    return pos + rng.uniform(-jitter, jitter, size=(n, 3))


def _spheres(n, radius, rho, pos, vel, crust, shape_index=0, material=0, system=None, id0=0):
    mass, inertia = sphere_mass_inertia(radius, rho)
    q = np.zeros((n, 4))
    q[:, 3] = 1.0
    return dict(id=np.arange(id0, id0 + n, dtype=np.int32), system=system,
                shape=np.full(n, shape_index, np.int32), material=np.full(n, material, np.int32),
                radius=np.asarray(radius, float), crust=np.full(n, crust), mass=mass, inertia=inertia,
                position=pos, quaternion=q, basis=None, velocity=vel, omega=np.zeros((n, 3)))


def settling_1k(n=1000, seed=0):
    """1,000 monodisperse spheres (r = 1 mm, rho = 2500) in a closed 20x20x60 mm
    box, jittered lattice (spacing 2.4 mm, +-0.1 mm), at rest, Hooke kn = 1e5,
    en = 0.9, mu = 0.5, kt = 0.8 kn, dt = 1e-5 s, 10,000 steps."""
    rng = np.random.default_rng(seed)
    crust = 0.05 * MM
    lo, hi = np.zeros(3), np.array([20.0, 20.0, 60.0]) * MM
    pos = lattice(n, lo, hi, 2.4 * MM, 1.2 * MM, 0.1 * MM, rng)
    r = np.full(n, 1.0 * MM)
    shapes = [(SPHERE, [1.0 * MM])]
    wshapes, obs = box_walls(lo, hi, "xXyYzZ", 0.5 * MM, crust, len(shapes), -1)
    shapes += wshapes
    kn = 1.0e5
    laws = [[(0, 0, HOOKE_MEMORY, hooke_memory_params(kn, 0.9, 0.5, 0.8 * kn)),
             (0, 1, HOOKE_MEMORY, hooke_memory_params(kn, 0.9, 0.5, 0.8 * kn))]]
    dom = [dict(origin=lo, size=hi - lo, cell_size=2.0 * 1.0 * MM, gravity=(0.0, 0.0, -9.81))]
    p = _spheres(n, r, 2500.0, pos, np.zeros((n, 3)), crust)
    return Scenario("settling_1k", shapes, dom, laws, [obs], p, 1.0e-5, 10000)


def polydisperse_200k(n=200_000, seed=1, vseed=2, height=370.0):
    """200,000 spheres, r ~ U[0.8, 1.2] mm, rho = 2500, floor + 4 side walls of
    a 100x100 mm box, lattice spacing 2.6 mm, velocities N(0, 0.05 m/s), same
    law as settling_1k, dt = 5e-6 s.  200k spheres do not fit a jittered
    cubic lattice in 100x100x200 mm, so the domain is 370 mm tall (the settled
    bed, about 145 mm, stays inside 200 mm)."""
    rng = np.random.default_rng(seed)
    vrng = np.random.default_rng(vseed)
    crust = 0.05 * MM
    lo, hi = np.zeros(3), np.array([100.0, 100.0, height]) * MM
    r = rng.uniform(0.8 * MM, 1.2 * MM, size=n)
    pos = lattice(n, lo, hi, 2.6 * MM, 1.3 * MM, 0.1 * MM, rng)
    vel = vrng.normal(0.0, 0.05, size=(n, 3))
    shapes = [(SPHERE, [1.0 * MM])]
    wshapes, obs = box_walls(lo, hi, "xXyYz", 0.5 * MM, crust, len(shapes), -1)
    shapes += wshapes
    kn = 1.0e5
    laws = [[(0, 0, HOOKE_MEMORY, hooke_memory_params(kn, 0.9, 0.5, 0.8 * kn)),
             (0, 1, HOOKE_MEMORY, hooke_memory_params(kn, 0.9, 0.5, 0.8 * kn))]]
    dom = [dict(origin=lo, size=hi - lo, cell_size=2.0 * 1.2 * MM, gravity=(0.0, 0.0, -9.81))]
    p = _spheres(n, r, 2500.0, pos, vel, crust)
    return Scenario("polydisperse_200k", shapes, dom, laws, [obs], p, 5.0e-6, 20000)


def ensemble_512(n_systems=512, seed=4, n_min=200, n_max=20000, dt=3.0e-6):
    """512 independent settling boxes: N_s log-uniform in [200, 20000],
    r ~ U[0.9, 1.1] mm, box w x w x 3w with w = 20 mm (N_s/1000)^(1/3), own
    kn ~ logU[5e4, 5e5], en ~ U[0.5, 0.95], mu ~ U[0.1, 0.8], kt = 0.8 kn.
    dt = 3e-6 s rather than the 5e-6 s of the specification: in dense packings
    the stiffest systems are unstable at 5e-6 s in the reference's own scheme
    (the oracle's system 57, kn = 4.9e5, en = 0.6, ends in a MotionError after
    4,500 steps and others heat up to 1 m/s), while all stay at rest-scale
    velocities at 3e-6 s."""
    rng = np.random.default_rng(seed)
    crust = 0.05 * MM
    ns = np.floor(np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=n_systems))).astype(int)
    shapes = [(SPHERE, [1.0 * MM])]
    doms, laws, obstacles, parts = [], [], [], []
    for s in range(n_systems):
        n = int(ns[s])
        w = 20.0 * MM * (n / 1000.0) ** (1.0 / 3.0)
        lo, hi = np.zeros(3), np.array([w, w, 3 * w])
        r = rng.uniform(0.9 * MM, 1.1 * MM, size=n)
        pos = lattice(n, lo, hi, 2.4 * MM, 1.2 * MM, 0.1 * MM, rng)
        wshapes, obs = box_walls(lo, hi, "xXyYzZ", 0.5 * MM, crust, len(shapes), -1)
        shapes += wshapes
        kn = math.exp(rng.uniform(math.log(5.0e4), math.log(5.0e5)))
        en = rng.uniform(0.5, 0.95)
        mu = rng.uniform(0.1, 0.8)
        laws.append([(0, 0, HOOKE_MEMORY, hooke_memory_params(kn, en, mu, 0.8 * kn)),
                     (0, 1, HOOKE_MEMORY, hooke_memory_params(kn, en, mu, 0.8 * kn))])
        doms.append(dict(origin=lo, size=hi - lo, cell_size=2.0 * 1.1 * MM, gravity=(0.0, 0.0, -9.81)))
        obstacles.append(obs)
        parts.append(_spheres(n, r, 2500.0, pos, np.zeros((n, 3)), crust, system=np.full(n, s, np.int32)))
    p = {k: (np.concatenate([q[k] for q in parts]) if parts[0][k] is not None else None) for k in parts[0]}
    return Scenario("ensemble_512", shapes, doms, laws, obstacles, p, dt, 5000, meta=dict(sizes=ns))


def adjoint_4k(seed=5, vseed=6, kn=1.0e5, en=0.9, mu=0.5, n=4096, kt_ratio=0.8):
    """4,096 spheres r = 1 mm on a 16^3 lattice (spacing 2.4 mm) in a
    40x40x60 mm box with floor + 4 walls, velocities N(0, 0.2 m/s); kn = 1e5,
    en = 0.9, mu = 0.5, kt = 0.8 kn, dt = 1e-5 s, 2,000 steps.  A smaller n
    keeps the first n lattice sites (the lowest layers)."""
    rng = np.random.default_rng(seed)
    vrng = np.random.default_rng(vseed)
    crust = 0.05 * MM
    lo, hi = np.zeros(3), np.array([40.0, 40.0, 60.0]) * MM
    pos = lattice(n, lo, hi, 2.4 * MM, 1.2 * MM, 0.1 * MM, rng)
    vel = vrng.normal(0.0, 0.2, size=(n, 3))
    shapes = [(SPHERE, [1.0 * MM])]
    wshapes, obs = box_walls(lo, hi, "xXyYz", 0.5 * MM, crust, len(shapes), -1)
    shapes += wshapes
    laws = [[(0, 0, HOOKE_MEMORY, hooke_memory_params(kn, en, mu, kt_ratio * kn)),
             (0, 1, HOOKE_MEMORY, hooke_memory_params(kn, en, mu, kt_ratio * kn))]]
    dom = [dict(origin=lo, size=hi - lo, cell_size=2.0 * 1.0 * MM, gravity=(0.0, 0.0, -9.81))]
    p = _spheres(n, np.full(n, 1.0 * MM), 2500.0, pos, vel, crust)
    return Scenario("adjoint_4k" if n == 4096 else "adjoint_%d" % n, shapes, dom, laws, [obs], p, 1.0e-5, 2000)


def small_box(n=64, seed=0, velocity_sigma=0.05, spacing=2.04, jitter=0.02, radius_range=(1.0, 1.0)):
    """A small dense cluster near the floor of a closed box (many contacts in
    the first steps) for parity tests that the oracle finishes in seconds."""
    rng = np.random.default_rng(seed)
    crust = 0.05 * MM
    side = max(8.0, math.ceil((n ** (1.0 / 3.0)) * spacing + 3.0))
    lo, hi = np.zeros(3), np.array([side, side, side * 1.5]) * MM
    r = rng.uniform(radius_range[0] * MM, radius_range[1] * MM, size=n)
    pos = lattice(n, lo, hi, spacing * MM, (radius_range[1] + jitter + 0.01) * MM, jitter * MM, rng)
    vel = rng.normal(0.0, velocity_sigma, size=(n, 3))
    shapes = [(SPHERE, [1.0 * MM])]
    wshapes, obs = box_walls(lo, hi, "xXyYzZ", 0.5 * MM, crust, len(shapes), -1)
    shapes += wshapes
    kn = 1.0e5
    laws = [[(0, 0, HOOKE_MEMORY, hooke_memory_params(kn, 0.9, 0.5, 0.8 * kn)),
             (0, 1, HOOKE_MEMORY, hooke_memory_params(kn, 0.9, 0.5, 0.8 * kn))]]
    dom = [dict(origin=lo, size=hi - lo, cell_size=2.0 * radius_range[1] * MM, gravity=(0.0, 0.0, -9.81))]
    p = _spheres(n, r, 2500.0, pos, vel, crust)
    return Scenario("small_box", shapes, dom, laws, [obs], p, 1.0e-5, 100)


def pressed_box(n=125, seed=5, force=0.05, mass=1.0e-5, vmax=1.0, gap=0.3 * MM, convex=False):
    """small_box whose lid (the upper z wall, id -6) is lowered to `gap` above
    the highest particle and driven by an imposed force (0, 0, force)
    (ObstacleImposedForce "ConstantTranslation"; the imposed force is the
    contact force the lid is to receive, upwards for a lid on a bed): it moves
    down at Vmax until the particles push back, then a PID controller drives
    the contact force on it towards the imposed force.  convex: the cubes,
    cylinders and octahedra of convex_box instead of spheres."""
    sc = convex_box(n, seed=seed, velocity_sigma=0.0) if convex else small_box(n, seed=seed, velocity_sigma=0.0)
    top = float(np.max(sc.particles["position"][:, 2] + sc.particles["radius"]))
    lid = dict(sc.obstacles[0][5])
    t = list(lid["transform"])
    thickness = 0.5 * MM
    t[11] = top + gap + thickness / 2.0
    lid["transform"] = t
    sc.obstacles[0][5] = lid
    sc.meta["loadings"] = [[dict(obstacle_id=lid["id"], type=5, t_start=0.0, t_end=1.0e9, vector=(0.0, 0.0, force),
                                 amplitude=(mass, vmax))]]
    sc.name = "pressed_box"
    return sc


def dense_cluster(n=343, seed=0, overlap=0.5e-6, velocity_sigma=0.02, radius=1.0 * MM):
    """Spheres on a cubic lattice whose spacing is 2r - overlap, so that every
    lattice neighbour pair (and the outer layer with the walls) starts in
    contact; small random velocities give tangential motion."""
    rng = np.random.default_rng(seed)
    crust = 0.05 * MM
    spacing = 2 * radius - overlap
    side_n = int(math.ceil(n ** (1.0 / 3.0)))
    inner = (side_n - 1) * spacing + 2 * radius - overlap
    lo = np.zeros(3)
    hi = np.array([inner, inner, inner * 1.5])
    k = np.arange(n)
    ix, iy, iz = k % side_n, (k // side_n) % side_n, k // (side_n * side_n)
    pos = np.stack([radius - overlap / 2 + ix * spacing, radius - overlap / 2 + iy * spacing,
                    radius - overlap / 2 + iz * spacing], 1)
    pos += rng.uniform(-0.2 * overlap, 0.2 * overlap, size=(n, 3))
    vel = rng.normal(0.0, velocity_sigma, size=(n, 3))
    r = np.full(n, radius)
    shapes = [(SPHERE, [radius])]
    wshapes, obs = box_walls(lo, hi, "xXyYzZ", 0.5 * MM, crust, len(shapes), -1)
    shapes += wshapes
    kn = 1.0e5
    laws = [[(0, 0, HOOKE_MEMORY, hooke_memory_params(kn, 0.9, 0.5, 0.8 * kn)),
             (0, 1, HOOKE_MEMORY, hooke_memory_params(kn, 0.9, 0.5, 0.8 * kn))]]
    dom = [dict(origin=lo, size=hi - lo, cell_size=2.0 * radius, gravity=(0.0, 0.0, -9.81))]
    p = _spheres(n, r, 2500.0, pos, vel, crust)
    return Scenario("dense_cluster", shapes, dom, laws, [obs], p, 1.0e-5, 100)


def octahedron(a):
    """Regular octahedron of circumradius a in the polyhedron parameter
    layout: nv, vertices, nf, then (k, indices) per face, outward-oriented."""
    v = [a, 0, 0, -a, 0, 0, 0, a, 0, 0, -a, 0, 0, 0, a, 0, 0, -a]
    faces = [[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4], [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]]
    return [6] + v + [8] + sum([[3] + f for f in faces], [])


def _tetra(a, b, c):
    """Volume and principal second moments (x, y, z axes) of the tetrahedron
    (0, a, b, c) (F. Tonon, J. Math. Stat. 1(1), 2004)."""
    x = [0.0, a[0], b[0], c[0]]
    y = [0.0, a[1], b[1], c[1]]
    z = [0.0, a[2], b[2], c[2]]
    det = abs(x[1] * y[2] * z[3] + y[1] * z[2] * x[3] + z[1] * x[2] * y[3]
              - z[1] * y[2] * x[3] - x[1] * z[2] * y[3] - y[1] * x[2] * z[3])
    def sq(u):
        return (u[0] * u[0] + u[0] * u[1] + u[1] * u[1] + u[0] * u[2] + u[1] * u[2] + u[2] * u[2]
                + u[0] * u[3] + u[1] * u[3] + u[2] * u[3] + u[3] * u[3])
    return det / 6.0, np.array([det * (sq(y) + sq(z)) / 60.0, det * (sq(x) + sq(z)) / 60.0,
                                det * (sq(x) + sq(y)) / 60.0])


def shape_volume_inertia(shape_type, params):
    """Volume and principal inertia per unit density of a shape, following the
    reference's BuildInertia / getVolume formulas."""
    if shape_type == SPHERE:
        r = params[0]
        return 4.0 * PI * math.pow(r, 3.0) / 3.0, np.full(3, 8.0 * PI * math.pow(r, 5.0) / 15.0)
    if shape_type == BOX:
        e = [abs(x) / 2.0 for x in params[:3]]
        v = 8.0 * e[0] * e[1] * e[2]
        return v, np.array([v * (e[1] ** 2 + e[2] ** 2) / 3.0, v * (e[0] ** 2 + e[2] ** 2) / 3.0,
                            v * (e[1] ** 2 + e[0] ** 2) / 3.0])
    if shape_type == CYLINDER:
        r, hh = params[0], params[1] / 2.0
        cst = 0.5 * hh * r * r * PI
        i0 = cst * (4.0 * hh * hh / 3.0 + r * r)
        return 2 * hh * PI * r * r, np.array([i0, 2.0 * cst * r * r, i0])
    nv = int(params[0])
    vert = np.array(params[1:1 + 3 * nv]).reshape(nv, 3)
    k = 1 + 3 * nv
    nf = int(params[k])
    k += 1
    vol, inertia = 0.0, np.zeros(3)
    for _ in range(nf):
        m = int(params[k])
        f = [int(t) for t in params[k + 1:k + 1 + m]]
        k += 1 + m
        for j in range(1, m - 1):
            dv, di = _tetra(vert[f[0]], vert[f[j]], vert[f[j + 1]])
            vol += dv
            inertia += di
    return vol, inertia


def circumscribed_radius(shape_type, params):
    if shape_type == SPHERE:
        return params[0]
    if shape_type == BOX:
        return math.sqrt(sum((abs(x) / 2.0) ** 2 for x in params[:3]))
    if shape_type == CYLINDER:
        return math.sqrt(params[0] ** 2 + (params[1] / 2.0) ** 2)
    nv = int(params[0])
    vert = np.array(params[1:1 + 3 * nv]).reshape(nv, 3)
    return float(np.sqrt(np.max(np.sum(vert * vert, axis=1))))


def random_quaternions(n, rng):
    """Uniform random unit quaternions (K. Shoemake, "Uniform random
    rotations", Graphics Gems III, 1992), xyzw."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    q = np.stack([a * np.sin(2 * PI * u2), a * np.cos(2 * PI * u2), b * np.sin(2 * PI * u3),
                  b * np.cos(2 * PI * u3)], 1)
    return q


def quaternion_basis(q):
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    return np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                     2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                     2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], 1)


CONVEX_SHAPES = [(BOX, [2.0 * MM, 2.0 * MM, 2.0 * MM]), (CYLINDER, [1.0 * MM, 2.0 * MM]),
                 (POLYHEDRON, octahedron(1.2 * MM))]
CONVEX_FRACTIONS = [0.4, 0.3, 0.3]


def _convex_particles(pos, rng, rho=2500.0, crust=0.05 * MM, fractions=CONVEX_FRACTIONS, shape_offset=0):
    n = len(pos)
    kinds = rng.choice(len(CONVEX_SHAPES), size=n, p=fractions)
    q = random_quaternions(n, rng)
    mass = np.zeros(n)
    inertia = np.zeros((n, 3))
    radius = np.zeros(n)
    for k, (t, prm) in enumerate(CONVEX_SHAPES):
        vol, inr = shape_volume_inertia(t, prm)
        sel = kinds == k
        mass[sel] = rho * vol
        inertia[sel] = inr * rho
        radius[sel] = circumscribed_radius(t, prm)
    return dict(id=np.arange(n, dtype=np.int32), system=None, shape=(kinds + shape_offset).astype(np.int32),
                material=np.zeros(n, np.int32), radius=radius, crust=np.full(n, crust), mass=mass,
                inertia=inertia, position=pos, quaternion=q, basis=quaternion_basis(q),
                velocity=np.zeros((n, 3)), omega=np.zeros((n, 3)))


def convex_box(n=216, seed=0, spacing=3.6, jitter=0.05, velocity_sigma=0.2, kn=2.0e5, en=0.7, mu=0.4,
               converge_time=None):
    """Cubes, cylinders and octahedra (40/30/30 %) with random orientations on
    a jittered lattice in a closed box: the static-wall counterpart of the
    rotating-drum workload, for parity tests of the GJK narrowphase.  With
    `converge_time` T every particle also moves towards the box centre at
    (centre - x) / T, so the lattice collapses into a dense cluster after
    about T."""
    rng = np.random.default_rng(seed)
    crust = 0.05 * MM
    side_n = int(math.ceil(n ** (1.0 / 3.0)))
    rmax = max(circumscribed_radius(t, p) for t, p in CONVEX_SHAPES)
    lo = np.zeros(3)
    side = (side_n - 1) * spacing * MM + 2 * (rmax * 1.0 + 0.3 * MM) + 0.0
    hi = np.array([side, side, side * 1.2])
    pos = lattice(n, lo, hi, spacing * MM, rmax + 0.2 * MM, jitter * MM, rng)
    p = _convex_particles(pos, rng, crust=crust)
    p["velocity"] = rng.normal(0.0, velocity_sigma, size=(n, 3))
    if converge_time:
        p["velocity"] += (0.5 * (lo + hi) - pos) / converge_time
    p["omega"] = rng.normal(0.0, 50.0, size=(n, 3))
    shapes = list(CONVEX_SHAPES)
    wshapes, obs = box_walls(lo, hi, "xXyYzZ", 0.5 * MM, crust, len(shapes), -1)
    shapes += wshapes
    laws = [[(0, 0, HOOKE_MEMORY, hooke_memory_params(kn, en, mu, 0.8 * kn)),
             (0, 1, HOOKE_MEMORY, hooke_memory_params(kn, en, mu, 0.8 * kn))]]
    dom = [dict(origin=lo, size=hi - lo, cell_size=2.0 * rmax, gravity=(0.0, 0.0, -9.81))]
    return Scenario("convex_box", shapes, dom, laws, [obs], p, 2.0e-6, 100)


def drum(n=100_000, seed=3, radius=110.0 * MM, length=147.0 * MM, n_boxes=64, rpm=30.0, width=5.0 * MM,
         spacing=3.7 * MM, initial_velocity=(0.0, 0.0, 0.0)):
    """Cubes (edge 2 mm), cylinders (r 1 mm, h 2 mm) and regular octahedra
    (circumradius 1.2 mm), 40/30/30 %, random orientations, in a drum whose
    shell is n_boxes boxes on a circle (CylindricalShell with box elements,
    CylindricalShell.cpp:12-100) closed by two end plates, rotating about its
    axis (z) at `rpm`.  kn = 2e5, en = 0.7, mu = 0.4, kt = 0.8 kn,
    dt = 2e-6 s.  100k such particles do not fit a 60 mm x 80 mm drum (the
    particles alone are ~64 % of its volume), so the drum is 110 mm x 147 mm
    (same L/R)."""
    rng = np.random.default_rng(seed)
    crust = 0.05 * MM
    rmax = max(circumscribed_radius(t, p) for t, p in CONVEX_SHAPES)
    # lattice sites inside the drum
    m = int((2 * radius) / spacing) + 1
    g = (np.arange(m) - (m - 1) / 2.0) * spacing
    zs = np.arange(rmax + 0.5 * MM, length - rmax - 0.5 * MM, spacing)
    X, Y, Z = np.meshgrid(g, g, zs, indexing="ij")
    sites = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    sites = sites[np.hypot(sites[:, 0], sites[:, 1]) < radius - rmax - 0.5 * MM]
    order = np.lexsort((sites[:, 0], sites[:, 2], sites[:, 1]))   # bottom (y) first
    sites = sites[order]
    if len(sites) < n:
        raise ValueError("drum holds %d lattice sites < %d" % (len(sites), n))
    pos = sites[:n] + rng.uniform(-0.1 * MM, 0.1 * MM, size=(n, 3))
    p = _convex_particles(pos, rng, crust=crust)
    p["velocity"] += np.asarray(initial_velocity, dtype=np.float64)
    shapes = list(CONVEX_SHAPES)
    omega = (0.0, 0.0, rpm * 2.0 * PI / 60.0)
    centre = (0.0, 0.0, 0.5 * length)
    delta = 2.0 * PI / n_boxes
    ly = 2.0 * (radius + width) * (math.sin(delta) - (1.0 - math.cos(delta)) / math.tan(delta))
    obs = []
    shapes.append((BOX, [width, ly, length + 2 * width]))
    shell = len(shapes) - 1
    ext_r = radius + width / 2.0
    for i in range(n_boxes):
        ang = (0.5 + i) * delta
        c, s_ = math.cos(ang), math.sin(ang)
        obs.append(dict(id=-1 - i, shape=shell, material=1, crust=crust, moving=1,
                        transform=[c, -s_, 0, s_, c, 0, 0, 0, 1, ext_r * c, ext_r * s_, 0.5 * length],
                        omega=omega, rotation_center=centre))
    shapes.append((BOX, [2 * (radius + width), 2 * (radius + width), width]))
    cap = len(shapes) - 1
    for k, zc in enumerate([-width / 2.0, length + width / 2.0]):
        obs.append(dict(id=-1 - n_boxes - k, shape=cap, material=1, crust=crust, moving=1,
                        transform=[1, 0, 0, 0, 1, 0, 0, 0, 1, 0.0, 0.0, zc], omega=omega,
                        rotation_center=centre))
    kn = 2.0e5
    laws = [[(0, 0, HOOKE_MEMORY, hooke_memory_params(kn, 0.7, 0.4, 0.8 * kn)),
             (0, 1, HOOKE_MEMORY, hooke_memory_params(kn, 0.7, 0.4, 0.8 * kn))]]
    lo = np.array([-radius - 1.0 * MM, -radius - 1.0 * MM, 0.0])
    dom = [dict(origin=lo, size=np.array([2 * radius + 2.0 * MM, 2 * radius + 2.0 * MM, length]),
                cell_size=2.0 * rmax, gravity=(0.0, -9.81, 0.0))]
    return Scenario("drum_100k", shapes, dom, laws, [obs], p, 2.0e-6, 10000)


def apply(sim, sc):
    """Registers shapes, domains, laws and obstacles of `sc` on `sim` and
    uploads the particles.  Returns the shape-id map."""
    ids = setup(sim, sc)
    p = dict(sc.particles)
    p["shape"] = np.asarray(ids, np.int32)[np.asarray(p["shape"])]
    sim.upload(p)
    return ids


def setup(sim, sc):
    """Everything of `apply` but the particle upload: shapes, collision
    options, domains, laws, obstacles and their loadings.  Returns the
    shape-id map (scenario shape index -> registered shape id)."""
    ids = [sim.add_shape(t, prm) for t, prm in sc.shapes]
    if sc.meta.get("collision") is not None:
        sim.set_collision_algorithm(sc.meta["collision"])
    if sc.meta.get("collision_options"):
        # <CollisionDetection Tolerance Acceleration History>
        sim.set_collision_options(**sc.meta["collision_options"])
    for s, d in enumerate(sc.domains):
        sim.set_domain(s, d["origin"], d["size"], d["cell_size"], d["gravity"])
        for a, b, law, prm in sc.laws[s]:
            sim.set_contact_law(s, a, b, law, prm)
        obs = []
        for o in sc.obstacles[s]:
            o2 = dict(o)
            o2["shape"] = ids[o["shape"]]
            obs.append(o2)
        sim.set_obstacles(s, obs)
        loads = sc.meta.get("loadings")
        if loads and loads[s]:
            sim.set_obstacle_loadings(s, loads[s])
    return ids
