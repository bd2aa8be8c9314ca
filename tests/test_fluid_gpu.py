"""The DEM side of the fluid coupling on the CUDA path.

* Immersed particles (buoyant weight, coupling factor on the accelerations,
  the fluid's forces and torques): the FP64 CUDA path against the oracle,
  which tests/test_fluid_cpu.py holds to the reference itself; positions
  within 1e-13 m after 50 steps, spheres and convex bodies.
* The fluid step (GrainsCoupledWithFluid::Simulation): the DEM step count of
  each fluid step follows the reference's formula, carried over from call to
  call, and the state equals the same DEM steps taken directly.
* The export for the fluid solver (GrainsToFluid as GrainsToBasilisk passes
  it): the CUDA library's string against the reference's own objects and
  formatting on the same state, token for token.
* The fluid solvers' C interface (Init_Grains, Simu_Grains,
  UpdateVelocityGrains, GrainsToBasilisk, NumberOfRigidBodiesInBasilisk)
  driving an attached context equals the grains_gpu calls it stands for."""
import ctypes as C
import os

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, GrainsLib

from helpers import make

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")


def immersed(sc, seed):
    rng = np.random.default_rng(seed)
    w = float(np.mean(sc.particles["mass"])) * 9.81
    return (np.full(sc.n, 2500.0), rng.normal(0.0, 0.3 * w, size=(sc.n, 3)),
            rng.normal(0.0, 0.3 * w * 1e-3, size=(sc.n, 3)))


def case(name):
    return S.small_box(125, seed=9, velocity_sigma=0.2) if name == "spheres" else S.convex_box(64, seed=4)


@pytest.mark.parametrize("corrected", [True, False], ids=["corrected", "uncorrected"])
@pytest.mark.parametrize("name", ["spheres", "convex"])
def test_immersed_particles_follow_the_oracle(oracle_lib, gpu_lib, name, corrected):
    sc = case(name)
    rho, force, torque = immersed(sc, 1)
    out = []
    for lib in (oracle_lib, gpu_lib):
        s = make(lib, sc, FP64)
        if lib is oracle_lib:
            s.set_polyhedron_support(2)
        s.set_fluid(1000.0, corrected, rho)
        s.set_hydro_forces(force, torque)
        s.initialize_leapfrog(0.0, sc.dt)
        s.step(50, 0.0, sc.dt)
        out.append(s.download())
        s.close()
    assert np.max(np.abs(out[0]["position"] - out[1]["position"])) < 1e-13
    assert np.max(np.abs(out[0]["velocity"] - out[1]["velocity"])) < 1e-9


def test_fluid_step_substeps(gpu_lib):
    sc = S.small_box(64, seed=3, velocity_sigma=0.1)
    a, b = make(gpu_lib, sc, FP64), make(gpu_lib, sc, FP64)
    for s in (a, b):
        s.initialize_leapfrog(0.0, sc.dt)
    ndt, t, counts, expected, n = 7, 0.0, [], [], 7
    for k in range(3):
        dtf = 1e-4 * (k + 1)
        ndt, t = a.fluid_step(dtf, 2e-6, 1e-5, ndt, t)
        counts.append(ndt)
        # GrainsCoupledWithFluid::Simulation (GrainsCoupledWithFluid.cpp:128-133)
        dteff = max(min(1e-5, dtf / n), 2e-6)
        n = int(dtf / dteff)
        expected.append(n)
    assert counts == expected
    tb = 0.0
    for k, n in enumerate(counts):
        tb = b.step(n, tb, 1e-4 * (k + 1) / n)
    assert abs(t - tb) < 1e-18
    assert np.array_equal(a.download()["position"], b.download()["position"])
    a.close()
    b.close()


def densities(tokens, n):
    """The density of every particle record of an export (token 9 of a
    record; records end after their envelope points and faces)."""
    out, k = [], 1
    for _ in range(n):
        out.append(float(tokens[k + 9]))
        k += 3 + 6 + 2 + 6 + 9 + 3 + 1
        npts = int(tokens[k])
        k += 1 + 3 * npts
        nf = int(tokens[k])
        k += 1
        for _f in range(nf):
            k += 1 + int(tokens[k])
    assert k == len(tokens)
    return np.array(out)


def ref_features(ref_lib, s):
    f = ref_lib.dll.grains_ref_fluid_features
    f.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(C.c_int64)]
    f.restype = C.c_int
    n = C.c_int64(0)
    assert f(s.ctx, None, 0, C.byref(n)) == 0
    buf = C.create_string_buffer(n.value)
    assert f(s.ctx, buf, n.value, C.byref(n)) == 0
    return buf.value.decode()


@pytest.mark.parametrize("name", ["spheres", "convex"])
def test_fluid_features_match_the_reference(gpu_lib, name):
    if not os.path.exists(REF_SO):
        pytest.skip("the reference library is not built (needs the reference sources)")
    ref_lib = GrainsLib(REF_SO, "grains_ref_")
    sc = case(name)
    rng = np.random.default_rng(2)
    sc.particles["omega"] = rng.normal(0.0, 30.0, size=(sc.n, 3))
    r = make(ref_lib, sc)
    g = make(gpu_lib, sc, FP64)
    a = ref_features(ref_lib, r).split()
    # the particle densities are input data (the reference input's class
    # densities): handed over with the fluid set-up, no fluid
    g.set_fluid(0.0, True, densities(a, sc.n))
    b = g.fluid_features().split()
    r.close()
    g.close()
    assert len(a) == len(b) and len(a) > 40 * sc.n // 2
    assert a[0] == str(sc.n)
    diff = [k for k, (x, y) in enumerate(zip(a, b)) if x != y]
    assert not diff, [(a[k], b[k]) for k in diff[:5]]


def test_basilisk_interface_drives_the_attached_context(gpu_lib):
    sc = S.small_box(64, seed=3, velocity_sigma=0.1)
    rho = np.full(sc.n, 2500.0)
    a, b = make(gpu_lib, sc, FP64), make(gpu_lib, sc, FP64)
    dll = gpu_lib.dll
    dll.grains_gpu_basilisk_attach.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int64]
    dll.Init_Grains.argtypes = [C.c_char_p, C.c_double, C.c_bool, C.c_bool]
    dll.Simu_Grains.argtypes = [C.c_double]
    dll.GrainsToBasilisk.argtypes = [C.POINTER(C.c_int)]
    dll.GrainsToBasilisk.restype = C.c_void_p
    dll.UpdateVelocityGrains.argtypes = [C.POINTER(C.POINTER(C.c_double)), C.c_int]
    dll.NumberOfRigidBodiesInBasilisk.argtypes = [C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    a.set_fluid(0.0, True, rho)  # the particle densities, before the interface applies the fluid
    assert dll.grains_gpu_basilisk_attach(a.ctx, 2e-6, 1e-5, 10) == 0
    dll.Init_Grains(b"unused.xml", 1000.0, False, True)
    b.set_fluid(1000.0, True, rho)
    b.initialize_leapfrog(0.0, 2e-6)
    # velocities from the fluid, rows by id
    rng = np.random.default_rng(4)
    v6 = rng.normal(0.0, 0.05, size=(sc.n, 6))
    rows = (C.POINTER(C.c_double) * sc.n)(*[np.ctypeslib.as_ctypes(v6[k]) for k in range(sc.n)])
    dll.UpdateVelocityGrains(rows, sc.n)
    order = np.argsort(sc.particles["id"])
    vel, om = np.zeros((sc.n, 3)), np.zeros((sc.n, 3))
    vel[order], om[order] = v6[:, :3], v6[:, 3:]
    b.set_velocities(vel, om)
    dll.Simu_Grains(5e-5)
    ndt, t = b.fluid_step(5e-5, 2e-6, 1e-5, 10, 0.0)
    np_, no_ = C.c_size_t(0), C.c_size_t(0)
    dll.NumberOfRigidBodiesInBasilisk(C.byref(np_), C.byref(no_))
    assert (np_.value, no_.value) == (sc.n, 0)
    size = C.c_int(0)
    ptr = dll.GrainsToBasilisk(C.byref(size))
    text = C.string_at(ptr, size.value - 1).decode()
    C.CDLL(None).free(C.c_void_p(ptr))
    assert text == b.fluid_features()
    assert np.array_equal(a.download()["position"], b.download()["position"])
    a.close()
    b.close()
