"""The Hertz and HertzMemory contact laws (HertzContactForceModel.cpp,
HertzMemoryContactForceModel.cpp) on the CUDA path against the CPU oracle,
which the reference fixtures hertz_dense125 and hertz_memory216_rolling pin.

Dense clusters, advanced by the oracle under the Hertz law until most lattice
neighbours touch, then one force evaluation and a short trajectory from the
same state on both sides.  Bars as for the Hooke laws: plain FP64 forces within
1e-12 relative (floor: the particle weight), mixed precision within 1e-5;
mixed torques within 3e-5 of the 1e-7 N m floor."""
import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED, GrainsError

from helpers import check_contact_forces, make, pair_set, rel_err

pytestmark = pytest.mark.gpu

ES, GS = 1.0e9, 0.3e9
DT = 2.0e-6


def hertz_cluster(oracle_lib, law, n=343, seed=11, steps=30, sigma=0.1):
    sc = S.dense_cluster(n, seed=seed, velocity_sigma=sigma)
    if law == S.HERTZ:
        prm = [ES, 0.8, 0.4, 1.0e-3, GS]
    else:
        prm = [ES, 0.8, 0.4, GS, 0.05, 0.3, 0.0]
    sc.laws = [[(a, b, law, prm) for a, b, _, _ in sc.laws[0]]]
    sc.dt = DT
    o = make(oracle_lib, sc)
    o.initialize_leapfrog(0.0, sc.dt)
    o.step(steps, 0.0, sc.dt)
    st = o.download()
    mem = o.contact_memory()
    p = dict(sc.particles)
    for k in ["position", "quaternion", "velocity", "omega"]:
        p[k] = st[k]
    sc.particles = p
    return sc, mem


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("law", [S.HERTZ, S.HERTZ_MEMORY], ids=["hertz", "hertz_memory"])
def test_one_force_evaluation(oracle_lib, gpu_lib, law, precision):
    sc, mem = hertz_cluster(oracle_lib, law)
    o, g = make(oracle_lib, sc), make(gpu_lib, sc, precision)
    o.upload_contact_memory(mem)
    g.upload_contact_memory(mem)
    o.compute_forces(0.0, sc.dt)
    g.compute_forces(0.0, sc.dt)
    do, dg = o.download(), g.download()
    assert int(do["coordination"].sum()) > 500
    assert np.array_equal(do["coordination"], dg["coordination"])
    weight = sc.particles["mass"][0] * 9.81
    assert rel_err(dg["force"], do["force"], weight) < (1e-12 if precision == FP64 else 1e-5)
    # mixed torques: a particle's torque is the sum of its contacts' tangential
    # torques (|lever| |F_t| ~ 1e-5 N m here), which nearly cancel, each
    # carrying FP32 rounding of 1e-7 of itself; against the 1e-7 N m floor that
    # is up to a few 1e-5
    assert rel_err(dg["torque"], do["torque"], weight * 1e-3) < (1e-10 if precision == FP64 else 3e-5)
    pg, fg = g.contact_forces()
    po, fo = o.contact_forces()
    assert np.array_equal(pg, po)
    check_contact_forces(fg, fo, weight, precision)
    if law == S.HERTZ_MEMORY:
        assert pair_set(o.contact_pairs()) == pair_set(g.contact_pairs())
        mo, mg = o.contact_memory(), g.contact_memory()
        ko = {(a, b): i for i, (a, b) in enumerate(zip(mo["owner"], mo["other"]))}
        kg = {(a, b): i for i, (a, b) in enumerate(zip(mg["owner"], mg["other"]))}
        assert set(ko) == set(kg)
        io = np.array([ko[k] for k in sorted(ko)])
        ig = np.array([kg[k] for k in sorted(ko)])
        tol = 1e-9 if precision == FP64 else 1e-4
        assert rel_err(mg["kdelta"][ig], mo["kdelta"][io], 1e-3 * weight) < tol
        assert rel_err(mg["spring_torque"][ig], mo["spring_torque"][io], 1e-6 * weight) < tol
        assert np.abs(mo["spring_torque"]).max() > 0, "the rolling spring should be loaded"


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("law", [S.HERTZ, S.HERTZ_MEMORY], ids=["hertz", "hertz_memory"])
def test_short_trajectory(oracle_lib, gpu_lib, law, precision):
    """20 KDK steps (graph-replayed on the device) from identical states."""
    sc, mem = hertz_cluster(oracle_lib, law, steps=20)
    o, g = make(oracle_lib, sc), make(gpu_lib, sc, precision)
    o.upload_contact_memory(mem)
    g.upload_contact_memory(mem)
    for s in (o, g):
        s.compute_forces(0.0, sc.dt)
        s.step(20, 0.0, sc.dt)
    do, dg = o.download(), g.download()
    assert np.max(np.abs(dg["position"] - do["position"])) < (1e-14 if precision == FP64 else 1e-10)
    assert np.max(np.abs(dg["velocity"] - do["velocity"])) < (1e-10 if precision == FP64 else 1e-5)
    assert np.max(np.abs(dg["omega"] - do["omega"])) < (1e-6 if precision == FP64 else 1e-2)


def test_hertz_parameters_are_checked(gpu_lib):
    sc = S.dense_cluster(27, seed=1)
    g = make(gpu_lib, sc, FP64)
    with pytest.raises(GrainsError):
        g.set_contact_law(0, 0, 0, S.HERTZ, [ES, 0.8, 0.4, 1.0e-3])          # 4 of 5 parameters
    with pytest.raises(GrainsError):
        g.set_contact_law(0, 0, 0, S.HERTZ_MEMORY, [0.0, 0.8, 0.4, GS, 0.0, 0.0, 0.0])  # Es = 0
    g.close()
