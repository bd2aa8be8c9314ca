"""Parity of the CUDA path with the CPU oracle on identical states.

* candidate pairs and contact pairs: bit-exact sets (both decide in double
  with the reference's rounding);
* one force evaluation: plain FP64 forces / torques within 1e-12 relative,
  mixed precision within 1e-5 relative (force floor = the particle weight);
* short trajectories: FP64 states within tight absolute bounds.
"""
import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED

from helpers import check_contact_forces, make, pair_set, rel_err

pytestmark = pytest.mark.gpu


def evolved(oracle_lib, n=343, seed=1, steps=20, sigma=0.05):
    """A dense cluster advanced by the oracle: returns the scenario whose
    particle state (and contact memory) are the oracle's after `steps`."""
    sc = S.dense_cluster(n, seed=seed, velocity_sigma=sigma)
    o = make(oracle_lib, sc)
    o.initialize_leapfrog(0.0, sc.dt)
    o.step(steps, 0.0, sc.dt)
    st = o.download()
    mem = o.contact_memory()
    p = dict(sc.particles)
    for k in ["position", "quaternion", "basis", "velocity", "omega"]:
        p[k] = st[k]
    sc.particles = p
    return sc, mem


def both(oracle_lib, gpu_lib, sc, mem=None, precision=FP64):
    """The oracle (with the CUDA path's polyhedron support rule: a hill climb
    that every GJK run starts at vertex 0) and the CUDA path on the same
    scenario."""
    o = make(oracle_lib, sc)
    o.set_polyhedron_support(2)
    g = make(gpu_lib, sc, precision)
    if mem is not None:
        o.upload_contact_memory(mem)
        g.upload_contact_memory(mem)
    return o, g


@pytest.mark.parametrize("name", ["settling_1k", "small_box", "evolved"])
def test_candidate_pairs_bit_exact(oracle_lib, gpu_lib, name):
    if name == "settling_1k":
        sc = S.settling_1k()
    elif name == "small_box":
        sc = S.small_box(125, seed=7)
    else:
        sc, _ = evolved(oracle_lib)
    o, g = both(oracle_lib, gpu_lib, sc)
    co = o.candidate_pairs(include_obstacles=True)
    cg = g.candidate_pairs(include_obstacles=True)
    assert len(co) == len(cg)
    assert np.array_equal(co, cg)
    assert len(pair_set(co)) == len(co)


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_one_force_evaluation(oracle_lib, gpu_lib, precision):
    sc, mem = evolved(oracle_lib)
    o, g = both(oracle_lib, gpu_lib, sc, mem, precision)
    o.reset_stats()
    g.reset_stats()
    o.compute_forces(0.0, sc.dt)
    g.compute_forces(0.0, sc.dt)
    po, pg = o.contact_pairs(), g.contact_pairs()
    assert len(po) > 50, "the evolved state should have many contacts"
    assert pair_set(po) == pair_set(pg)
    so, sg = o.stats(), g.stats()
    assert so["n_contacts"] == sg["n_contacts"]
    assert so["n_obstacle_contacts"] == sg["n_obstacle_contacts"]
    do, dg = o.download(), g.download()
    assert np.array_equal(do["coordination"], dg["coordination"])
    weight = sc.particles["mass"][0] * 9.81
    tol = 1e-12 if precision == FP64 else 1e-5
    assert rel_err(dg["force"], do["force"], weight) < tol
    pg, fg = g.contact_forces()
    po, fo = o.contact_forces()
    assert np.array_equal(pg, po)
    check_contact_forces(fg, fo, weight, precision)
    torque_scale = weight * 1e-3
    assert rel_err(dg["torque"], do["torque"], torque_scale) < (1e-10 if precision == FP64 else 1e-5)
    # contact memory after the evaluation
    mo, mg = o.contact_memory(), g.contact_memory()
    ko = {(a, b): i for i, (a, b) in enumerate(zip(mo["owner"], mo["other"]))}
    kg = {(a, b): i for i, (a, b) in enumerate(zip(mg["owner"], mg["other"]))}
    assert set(ko) == set(kg)
    idx_o = np.array([ko[k] for k in sorted(ko)])
    idx_g = np.array([kg[k] for k in sorted(ko)])
    kscale = 1e-3 * weight
    assert rel_err(mg["kdelta"][idx_g], mo["kdelta"][idx_o], kscale) < (1e-9 if precision == FP64 else 1e-4)
    assert np.max(np.abs(mg["prev_normal"][idx_g] - mo["prev_normal"][idx_o])) < (1e-12 if precision == FP64 else 1e-6)


def test_move_and_advance_velocity_fp64(oracle_lib, gpu_lib):
    sc, mem = evolved(oracle_lib, steps=10)
    sc.particles["omega"] = np.random.default_rng(3).normal(0, 50.0, size=(sc.n, 3))
    o, g = both(oracle_lib, gpu_lib, sc, mem, FP64)
    for s in (o, g):
        s.compute_forces(0.0, sc.dt)
        s.move(0.0, 0.5 * sc.dt, sc.dt)
    do, dg = o.download(), g.download()
    assert np.max(np.abs(dg["position"] - do["position"])) < 1e-15
    assert np.max(np.abs(dg["velocity"] - do["velocity"])) < 1e-13
    assert np.max(np.abs(dg["quaternion"] - do["quaternion"])) < 1e-14
    assert np.max(np.abs(dg["omega"] - do["omega"])) < 1e-9
    for s in (o, g):
        s.link_update()
        s.compute_forces(sc.dt, sc.dt)
        s.advance_velocity(sc.dt, 0.5 * sc.dt)
    do, dg = o.download(), g.download()
    weight = sc.particles["mass"][0] * 9.81
    assert rel_err(dg["force"], do["force"], weight) < 1e-11
    assert np.max(np.abs(dg["velocity"] - do["velocity"])) < 1e-12


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_short_trajectory_matches_oracle(oracle_lib, gpu_lib, precision):
    """5 KDK steps of a dense cluster from identical states."""
    sc, mem = evolved(oracle_lib, steps=15)
    o, g = both(oracle_lib, gpu_lib, sc, mem, precision)
    for s in (o, g):
        s.compute_forces(0.0, sc.dt)
    o.step(5, 0.0, sc.dt)
    g.step(5, 0.0, sc.dt)
    do, dg = o.download(), g.download()
    assert np.max(np.abs(dg["position"] - do["position"])) < (1e-14 if precision == FP64 else 1e-10)
    assert np.max(np.abs(dg["velocity"] - do["velocity"])) < (1e-10 if precision == FP64 else 1e-5)


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_settling_statistics(oracle_lib, gpu_lib, precision):
    """Granular dynamics is chaotic (rounding differences grow by orders of
    magnitude per contact time), so long runs are compared statistically:
    256 spheres dropped into a box and left to settle for 9,000 steps; the
    bed height, the mean coordination and the (small) kinetic energy agree."""
    sc = S.settling_1k(256)
    o, g = make(oracle_lib, sc), make(gpu_lib, sc, precision)
    for s in (o, g):
        s.initialize_leapfrog(0.0, sc.dt)
        s.step(9000, 0.0, sc.dt)
    do, dg = o.download(), g.download()
    zo, zg = do["position"][:, 2].mean(), dg["position"][:, 2].mean()
    assert abs(zg - zo) < 0.02 * zo
    assert abs(dg["coordination"].mean() - do["coordination"].mean()) < 0.5
    m = sc.particles["mass"]
    ke = lambda d: 0.5 * float(np.sum(m * np.sum(d["velocity"] ** 2, axis=1)))
    ref_scale = float(np.sum(m)) * 9.81 * 1e-3   # potential energy of a 1 mm drop
    assert abs(ke(dg) - ke(do)) < 0.05 * ref_scale


def test_graph_steps_equal_single_steps(gpu_lib):
    """The CUDA-graph replay of the fused step gives the same bits as stepping
    one at a time through the per-phase entry points."""
    sc = S.dense_cluster(216, seed=11)
    a = make(gpu_lib, sc, FP64)
    b = make(gpu_lib, sc, FP64)
    for s in (a, b):
        s.initialize_leapfrog(0.0, sc.dt)
    ta = a.step(20, 0.0, sc.dt)
    tb = 0.0
    for _ in range(20):
        tb += sc.dt
        b.move(tb, 0.5 * sc.dt, sc.dt)
        b.link_update(tb, sc.dt)
        b.compute_forces(tb, sc.dt)
        b.advance_velocity(tb, 0.5 * sc.dt)
    da, db = a.download(), b.download()
    for k in ["position", "velocity", "omega", "quaternion", "force", "torque"]:
        assert np.array_equal(da[k], db[k]), k


def test_deterministic(gpu_lib):
    sc = S.dense_cluster(343, seed=5)
    outs = []
    for _ in range(2):
        g = make(gpu_lib, sc, MIXED)
        g.initialize_leapfrog(0.0, sc.dt)
        g.step(60, 0.0, sc.dt)
        outs.append(g.download())
    for k in ["position", "velocity", "force"]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def small_drum(n=300, converge_time=0.006):
    """The rotating drum at a test size: 300 cubes, cylinders and octahedra
    converging onto the shell bottom of a 25 mm x 30 mm drum of 32 boxes."""
    sc = S.drum(n=n, radius=25e-3, length=30e-3, n_boxes=32)
    target = np.array([0.0, -25e-3, 15e-3])
    sc.particles["velocity"] = sc.particles["velocity"] + (target - sc.particles["position"]) / converge_time
    return sc


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_rotating_obstacles_follow_the_oracle(oracle_lib, gpu_lib, precision):
    """Imposed rotation of the drum's 34 obstacles (ConstantRotation about the
    drum axis) over 400 steps, through the graph-captured step: poses within
    1e-14 m, i.e. a few units in the last place of the 0.03 m coordinates
    (the device's and the host's double sin/cos may differ in the last bit)."""
    sc = small_drum()
    o, g = both(oracle_lib, gpu_lib, sc, precision=precision)
    n_obs = len(sc.obstacles[0])
    t = 0.0
    for sim in (o, g):
        sim.initialize_leapfrog(0.0, sc.dt)
    for _ in range(4):
        to = o.step(100, t, sc.dt)
        t = g.step(100, t, sc.dt)
        assert t == to
        po, pg = o.obstacles(0, n_obs), g.obstacles(0, n_obs)
        assert np.max(np.abs(po - pg)) < 1e-14
    assert g.stats()["status"] == 0


def test_translating_obstacle_one_step_fp64(oracle_lib, gpu_lib):
    """A floor moving up (ConstantTranslation) under a dense cluster: forces
    of the first evaluations (obstacle velocity zero before the first move,
    then the imposed velocity) and the floor's position after 10 steps."""
    sc = S.dense_cluster(125, seed=1, velocity_sigma=0.0)
    floor = sc.obstacles[0][4]
    floor["moving"] = 1
    floor["velocity"] = [0.0, 0.0, 0.02]
    o, g = both(oracle_lib, gpu_lib, sc)
    weight = float(np.min(sc.particles["mass"])) * 9.81
    for sim in (o, g):
        sim.initialize_leapfrog(0.0, sc.dt)
    assert rel_err(g.download()["force"], o.download()["force"], weight) < 1e-12
    t = 0.0
    for _ in range(10):
        o.step(1, t, sc.dt)
        t = g.step(1, t, sc.dt)
        assert rel_err(g.download()["force"], o.download()["force"], weight) < 1e-9
    po, pg = o.obstacles(0, 6), g.obstacles(0, 6)
    assert np.max(np.abs(po - pg)) == 0.0
    assert pg[4, 11] > sc.obstacles[0][4]["transform"][11]


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_drum_contacts_match_oracle(oracle_lib, gpu_lib, precision):
    """The drum advanced by the oracle into a dense cluster against the shell,
    then one evaluation on both: pair sets identical, FP64 forces within
    1e-12, mixed within 1e-5 of the weight-floored force."""
    sc = small_drum()
    o = make(oracle_lib, sc)
    o.set_polyhedron_support(2)
    o.initialize_leapfrog(0.0, sc.dt)
    t = o.step(1500, 0.0, sc.dt)
    st = o.download()
    mem = o.contact_memory()
    n_obs = len(sc.obstacles[0])
    poses = o.obstacles(0, n_obs)
    p = dict(sc.particles)
    for k in ["position", "quaternion", "basis", "velocity", "omega"]:
        p[k] = st[k]
    sc.particles = p
    obs = [dict(ob) for ob in sc.obstacles[0]]
    for k, ob in enumerate(obs):
        ob["transform"] = list(poses[k])
        ob["rotation_center"] = list(ob["rotation_center"])
    sc.obstacles = [obs]
    o2, g = both(oracle_lib, gpu_lib, sc, mem, precision)
    o2.compute_forces(t, sc.dt)
    g.compute_forces(t, sc.dt)
    do, dg = o2.download(), g.download()
    assert pair_set(g.contact_pairs()) == pair_set(o2.contact_pairs())
    assert len(o2.contact_pairs()) > 100
    assert np.array_equal(dg["coordination"], do["coordination"])
    weight = float(np.min(sc.particles["mass"])) * 9.81
    # mixed: FP32 rounding of large face-contact forces that nearly cancel in a
    # particle's sum; every single contact force is held to 1e-5
    assert rel_err(dg["force"], do["force"], weight) < (1e-12 if precision == FP64 else 1e-4)
    pg, fg = g.contact_forces()
    po, fo = o2.contact_forces()
    assert np.array_equal(pg, po)
    check_contact_forces(fg, fo, weight, precision)


def test_grid_spanning_many_scan_tiles(oracle_lib, gpu_lib):
    """A dense cluster of 512 spheres in a corner of a 60 mm box: a grid of
    30 x 30 x 30 = 27,000 cells, over six 4,096-cell tiles of the cell-count
    scan (scan_tiles / scan_finish), so the finishing blocks add the totals of
    earlier tiles.  Against the oracle after 30 steps (FP64): candidate and
    contact pairs equal, states at rounding level, status clear; and the
    persistent launch (its own scan) gives the same bits."""
    sc = S.dense_cluster(512, seed=12, velocity_sigma=0.1)
    lo, hi = np.zeros(3), np.array([60.0, 60.0, 60.0]) * S.MM
    shapes = [sc.shapes[0]]
    wshapes, obs = S.box_walls(lo, hi, "xXyYzZ", 0.5 * S.MM, 0.05 * S.MM, len(shapes), -1)
    sc.shapes = shapes + wshapes
    sc.obstacles = [obs]
    sc.domains = [dict(sc.domains[0], origin=lo, size=hi - lo)]
    o, g = both(oracle_lib, gpu_lib, sc)
    assert np.array_equal(o.candidate_pairs(include_obstacles=True), g.candidate_pairs(include_obstacles=True))
    for s in (o, g):
        s.compute_forces(0.0, sc.dt)
    assert pair_set(g.contact_pairs()) == pair_set(o.contact_pairs())
    assert len(o.contact_pairs()) > 500
    weight = sc.particles["mass"][0] * 9.81
    assert rel_err(g.download()["force"], o.download()["force"], weight) < 1e-12
    runs = []
    for s in (o, g):
        s.initialize_leapfrog(0.0, sc.dt)
        t = s.step(30, 0.0, sc.dt)
        s.compute_forces(t, sc.dt)
        runs.append(s.download())
    assert pair_set(g.contact_pairs()) == pair_set(o.contact_pairs())
    assert np.max(np.abs(runs[1]["position"] - runs[0]["position"])) < 1e-13
    assert g.stats()["status"] == 0
    p = make(gpu_lib, sc, FP64)
    p.set_tuning(persistent=1)
    p.compute_forces(0.0, sc.dt)  # the same sequence as above
    p.initialize_leapfrog(0.0, sc.dt)
    t = p.step(30, 0.0, sc.dt)
    p.compute_forces(t, sc.dt)
    assert np.array_equal(p.download()["position"], runs[1]["position"])
