"""CPU checks of the C ABI: the CUDA library and the oracle load and export
every entry point declared in include/grains_gpu.h; host-side helpers agree
with the reference's geometry formulas.  No device code runs here."""
import math
import os
import re

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import BOX, CYLINDER, POLYHEDRON, SPHERE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "grains_gpu.h")
GPU_ONLY = {"get_stream", "synchronize", "launches_per_step", "set_barrier_test", "profile_kernels", "shape_properties",
            "sphere_contacts_noalloc", "adjoint_create", "adjoint_destroy", "adjoint_last_error",
            "adjoint_law_slots", "adjoint_forward", "adjoint_contact_signature", "adjoint_backward",
            "get_tuning", "set_tuning", "autotune", "reload_open", "reload_last_error", "reload_get",
            "reload_close", "format_double", "format_doubles", "basilisk_attach", "fluid_step", "fluid_features"}
# the fluid solvers' C interface (same names as the reference's
# InterfaceGrains3DBasilisk.h), exported by the CUDA library
BASILISK = ["Init_Grains", "Simu_Grains", "GrainsToBasilisk", "SetInitialTime", "SaveResults_Grains",
            "checkParaviewPostProcessing_Grains", "UpdateVelocityGrains", "SetInitialCycleNumber",
            "NumberOfRigidBodiesInBasilisk"]


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\bint\s+grains_gpu_(\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    for n in ["create", "destroy", "compute_forces", "move", "link_update", "advance_velocity", "step",
              "upload_particles", "download_particles", "get_candidate_pairs", "get_contact_pairs"]:
        assert n in names


def test_header_enums_match_the_python_binding():
    """Contact-law and shape codes of the header are the ones abi.py passes."""
    from pacific_b200 import abi
    txt = open(HEADER).read()
    for name in ["HOOKE", "HOOKE_MEMORY", "HERTZ", "HERTZ_MEMORY", "SPHERE", "BOX", "CYLINDER", "POLYHEDRON"]:
        m = re.search(r"\bGRAINS_GPU_%s\s*=\s*(\d+)" % name, txt)
        assert m and int(m.group(1)) == getattr(abi, name), name


def test_oracle_checks_hertz_parameters(oracle_lib):
    from pacific_b200.abi import GrainsError, HERTZ, HERTZ_MEMORY, FP64, Simulation
    sc = S.dense_cluster(8, seed=0)
    sim = Simulation(oracle_lib, FP64, max_particles=8)
    S.apply(sim, sc)
    sim.set_contact_law(0, 0, 0, HERTZ, [1e9, 0.8, 0.4, 1e-3, 0.3e9])
    sim.set_contact_law(0, 0, 0, HERTZ_MEMORY, [1e9, 0.8, 0.4, 0.3e9, 0.05, 0.3, 0.0])
    with pytest.raises(GrainsError):
        sim.set_contact_law(0, 0, 0, HERTZ, [1e9, 0.8, 0.4, 1e-3])
    with pytest.raises(GrainsError):
        sim.set_contact_law(0, 0, 0, HERTZ_MEMORY, [1e9, 0.8, 0.4, 0.3e9, 0.05, 0.3])
    sim.close()


def test_cuda_library_exports_every_declared_symbol():
    import ctypes
    import pacific_b200
    dll = ctypes.CDLL(pacific_b200.LIB_PATH)
    for n in declared():
        assert hasattr(dll, "grains_gpu_" + n), n
    txt = open(HEADER).read()
    for n in BASILISK:
        assert re.search(r"\b%s\s*\(" % n, txt), n
        assert hasattr(dll, n), n


def test_oracle_exports_the_same_contract(oracle_lib):
    import ctypes
    dll = ctypes.CDLL(oracle_lib.path)
    for n in declared():
        if n in GPU_ONLY:
            continue
        assert hasattr(dll, "grains_oracle_" + n), n


def test_shape_properties_match_reference_formulas():
    import pacific_b200
    gpu_lib = pacific_b200.load_library()
    r = 1.0e-3
    vol, circ, inertia = gpu_lib.shape_properties(SPHERE, [r])
    assert vol == 4.0 * math.pi * math.pow(r, 3.0) / 3.0
    assert circ == r
    assert np.all(inertia == 8.0 * math.pi * math.pow(r, 5.0) / 15.0)
    vol, circ, inertia = gpu_lib.shape_properties(BOX, [2e-3, 4e-3, 6e-3])
    e = np.array([1e-3, 2e-3, 3e-3])
    assert vol == pytest.approx(8 * e.prod(), rel=1e-15)
    assert circ == pytest.approx(np.linalg.norm(e), rel=1e-15)
    assert inertia[0] == pytest.approx(8 * e.prod() * (e[1] ** 2 + e[2] ** 2) / 3, rel=1e-14)
    vol, circ, inertia = gpu_lib.shape_properties(CYLINDER, [1e-3, 2e-3])
    assert vol == pytest.approx(2e-3 * math.pi * 1e-6, rel=1e-15)
    assert circ == pytest.approx(math.sqrt(2) * 1e-3, rel=1e-15)
    # regular octahedron of circumradius a: V = 4 a^3 / 3, I = 2/5 * (a^2/... ) m
    a = 1.2e-3
    verts = [a, 0, 0, -a, 0, 0, 0, a, 0, 0, -a, 0, 0, 0, a, 0, 0, -a]
    faces = [[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4], [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]]
    prm = [6] + verts + [8] + sum([[3] + f for f in faces], [])
    vol, circ, inertia = gpu_lib.shape_properties(POLYHEDRON, prm)
    assert vol == pytest.approx(4 * a ** 3 / 3, rel=1e-12)
    assert circ == pytest.approx(a, rel=1e-15)
    assert inertia[0] == pytest.approx(vol * a * a / 5, rel=1e-12)


def test_scenarios_are_valid():
    for sc in [S.settling_1k(), S.adjoint_4k(), S.small_box(100)]:
        p = sc.particles
        n = sc.n
        assert p["position"].shape == (n, 3)
        d = sc.domains[0]
        lo, hi = np.asarray(d["origin"]), np.asarray(d["origin"]) + np.asarray(d["size"])
        assert np.all(p["position"] - p["radius"][:, None] > lo)
        assert np.all(p["position"] + p["radius"][:, None] < hi)
    sc = S.settling_1k()
    assert sc.n == 1000 and sc.dt == 1e-5 and sc.n_steps == 10000
    assert np.allclose(sc.particles["mass"], 2500 * 4 / 3 * math.pi * 1e-9)


def test_polydisperse_lattice_has_no_initial_overlap():
    sc = S.polydisperse_200k(n=20_000)
    p = sc.particles
    # neighbours on the lattice are 2.6 mm apart; radii <= 1.2 mm and jitter <= 0.1 mm
    from scipy.spatial import cKDTree
    t = cKDTree(p["position"])
    pairs = t.query_pairs(2.41e-3, output_type="ndarray")
    if len(pairs):
        d = np.linalg.norm(p["position"][pairs[:, 0]] - p["position"][pairs[:, 1]], axis=1)
        assert np.all(d > p["radius"][pairs[:, 0]] + p["radius"][pairs[:, 1]])


def test_obstacle_loadings_are_checked(oracle_lib):
    from pacific_b200.abi import FP64, GrainsError, SIN_TRANSLATION, Simulation
    sc = S.dense_cluster(8, seed=0)
    sim = Simulation(oracle_lib, FP64, max_particles=8)
    S.apply(sim, sc)
    sim.set_obstacle_loadings(0, [dict(obstacle_id=-1, type=SIN_TRANSLATION, vector=(1, 0, 0), amplitude=0.1,
                                       period=1e-3)])
    with pytest.raises(GrainsError):
        sim.set_obstacle_loadings(0, [dict(obstacle_id=-99, type=SIN_TRANSLATION, vector=(1, 0, 0))])
    with pytest.raises(GrainsError):
        sim.set_obstacle_loadings(0, [dict(obstacle_id=-1, type=17, vector=(1, 0, 0))])
    sim.close()
