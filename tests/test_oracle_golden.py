"""Pins the CPU oracle to the reference: golden fixtures produced by the
reference Grains3D built from its own sources (tests/golden/make_golden.py)
are replayed through the oracle on identical states and memories.

Bars: contact / candidate pair sets and coordination numbers identical;
forces and torques within 1e-13 relative (floor: the particle weight);
states after the KDK steps within 1e-14 m / 1e-10 m/s / 1e-11 in the
quaternion components, forces then within 1e-8.  (Rolling resistance and the
flat-face contacts of convex bodies amplify last-bit differences of the force
sums over the steps: the reference's own continuing run and its replay of the
same recorded state differ by 1.1e-12 in quaternions and 1.1e-9 in forces after
the 20 steps of dense216_rolling.)"""
import glob
import json
import os

import numpy as np
import pytest

from helpers import make, pair_set, rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
# state fixtures (io_*.npz hold reference-written files, tests/test_io_*.py)
CASES = sorted(c for c in glob.glob(os.path.join(HERE, "golden", "*.npz"))
               if not os.path.basename(c).startswith("io_") and not c.endswith("_stats.npz"))


def load(path):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import golden_io as G
    z = np.load(path)
    return G, z, G.scenario_from_npz(z)


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def test_oracle_matches_reference_fixture(oracle_lib, path):
    G, z, sc = load(path)
    sim = make(oracle_lib, sc)
    sim.upload_contact_memory(G.memory_from(z, "mem_in_"))
    t = float(z["time"])
    sim.compute_forces(t, sc.dt)
    d = sim.download()
    weight = float(np.min(sc.particles["mass"])) * 9.81
    assert np.array_equal(d["coordination"], z["coordination"])
    assert np.array_equal(sim.candidate_pairs(), z["candidate_pairs"])
    if bool(z["has_contact_pairs"]):
        assert pair_set(sim.contact_pairs()) == pair_set(z["contact_pairs"])
    assert rel_err(d["force"], z["force"], weight) < 1e-13
    assert rel_err(d["torque"], z["torque"], weight * 1e-3) < 1e-12
    mo = G.memory_from(z, "mem_out_")
    m = sim.contact_memory()
    assert set(zip(m["owner"].tolist(), m["other"].tolist())) == set(zip(mo["owner"].tolist(), mo["other"].tolist()))
    steps = int(z["after_steps"])
    sim.step(steps, t, sc.dt)
    d = sim.download()
    assert np.max(np.abs(d["position"] - z["after_position"])) < 1e-14
    assert np.max(np.abs(d["velocity"] - z["after_velocity"])) < 1e-10
    assert np.max(np.abs(d["quaternion"] - z["after_quaternion"])) < 1e-11
    if "after_obstacles" in z.files:  # imposed obstacle motions (every kind, time windows)
        assert np.max(np.abs(sim.obstacles(0, len(sc.obstacles[0])) - z["after_obstacles"])) < 1e-15
    assert rel_err(d["force"], z["after_force"], weight) < 1e-8


def test_fixtures_exercise_the_path():
    """The fixture set covers particle-particle and wall contacts, memory,
    rolling friction, the memory-less Hooke law, the Hertz and HertzMemory
    laws, polydispersity, boxes, cylinders and polyhedra through the GJK
    narrowphase, and a rotating drum."""
    names = [os.path.basename(c)[:-4] for c in CASES]
    for n in ["dense125", "dense216_rolling", "poly_box200", "hooke_dense125", "settling_1k", "convex216",
              "drum300", "hertz_dense125", "hertz_memory216_rolling", "loadings125", "convex216_gjk_sv"]:
        assert n in names
    z = np.load(os.path.join(HERE, "golden", "convex216_gjk_sv.npz"))
    assert json.loads(str(z["spec"]))["collision"] == 1  # the signed-volume GJK
    z = np.load(os.path.join(HERE, "golden", "loadings125.npz"))
    types = {l["type"] for l in json.loads(str(z["spec"]))["loadings"][0]}
    assert types == {0, 1, 2, 3, 4}
    for n, law in [("hertz_dense125", 2), ("hertz_memory216_rolling", 3)]:
        z = np.load(os.path.join(HERE, "golden", n + ".npz"))
        assert {l[2] for l in json.loads(str(z["spec"]))["laws"][0]} == {law}
        assert int(z["coordination"].sum()) > 400 and np.abs(z["torque"]).max() > 0
    z = np.load(os.path.join(HERE, "golden", "dense125.npz"))
    assert len(z["contact_pairs"]) > 100 and len(z["mem_in_owner"]) > 100
    z = np.load(os.path.join(HERE, "golden", "convex216.npz"))
    shapes = {s[0] for s in json.loads(str(z["spec"]))["shapes"]}
    assert {1, 2, 3} <= shapes and len(z["contact_pairs"]) > 40
    # the drum: a rotating shell of boxes, with particle-obstacle contact memory
    z = np.load(os.path.join(HERE, "golden", "drum300.npz"))
    obstacles = json.loads(str(z["spec"]))["obstacles"][0]
    assert sum(o["moving"] for o in obstacles) == len(obstacles) > 30
    assert np.any(z["mem_in_owner"] < 0) or np.any(z["mem_in_other"] < 0)


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def test_polyhedron_support_rules(oracle_lib, path):
    """Polyhedron::support (Polyhedron.cpp:265-293) hill-climbs from a vertex
    each body keeps between calls.  The CUDA path's rule, a climb that every
    GJK run starts at vertex 0 (oracle mode 2), gives the reference's forces
    and the positions after the fixture's steps exactly on every fixture; the
    order-independent arg-max (mode 1) does so only without polyhedra, and
    stays within 2e-3 of the weight-floored force where flat polyhedron faces
    touch."""
    G, z, sc = load(path)
    poly = any(sh[0] == 3 for sh in sc.shapes)
    weight = float(np.min(sc.particles["mass"])) * 9.81
    for mode in (2, 1):
        sim = make(oracle_lib, sc)
        sim.set_polyhedron_support(mode)
        sim.upload_contact_memory(G.memory_from(z, "mem_in_"))
        t = float(z["time"])
        sim.compute_forces(t, sc.dt)
        d = sim.download()
        assert np.array_equal(d["coordination"], z["coordination"])
        if bool(z["has_contact_pairs"]):
            assert pair_set(sim.contact_pairs()) == pair_set(z["contact_pairs"])
        err = rel_err(d["force"], z["force"], weight)
        if mode == 2 or not poly:
            assert err < 1e-13
            sim.step(int(z["after_steps"]), t, sc.dt)
            assert np.max(np.abs(sim.download()["position"] - z["after_position"])) < 1e-13
        else:
            assert 0 < err < 2e-3
        sim.close()
