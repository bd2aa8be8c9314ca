#!/usr/bin/env python
"""Generates the golden fixtures of tests/golden/*.npz by running the
reference Grains3D itself (oracle/_ref/libgrains_ref.so, built from the
reference sources by oracle/ref/Makefile) on seeded scenarios.

Each case: the reference advances a scenario for `warm` steps (building up
contact memory) and its state and memory are recorded as the input.  A fresh
reference context then replays that input: one force evaluation (forces,
torques, coordination, contact and candidate pairs, memory) and `steps`
further KDK steps (positions, velocities, quaternions, angular velocities) are
recorded as the expected output.  Each of the two runs has its own process
because the reference keeps process-wide static state.

    python tests/golden/make_golden.py            # all cases
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")

CASES = {
    # name: (generator call, warm steps, steps after)
    "dense125": ("S.dense_cluster(125, seed=1, velocity_sigma=0.05)", 10, 20),
    "dense216_rolling": ("rolling(S.dense_cluster(216, seed=2, velocity_sigma=0.1))", 8, 20),
    "poly_box200": ("S.small_box(200, seed=3, velocity_sigma=0.3, spacing=2.45, jitter=0.02, "
                    "radius_range=(0.8, 1.2))", 400, 40),
    "hooke_dense125": ("hooke(S.dense_cluster(125, seed=4, velocity_sigma=0.1))", 5, 20),
    "settling_1k": ("S.settling_1k()", 1000, 30),
    "convex216": ("S.convex_box(216, seed=0, converge_time=0.004, velocity_sigma=0.05)", 900, 5),
    "drum300": ("converge(S.drum(n=300, radius=25e-3, length=30e-3, n_boxes=32), (0.0, -25e-3, 15e-3), 0.006)",
                1500, 3),
    "hertz_dense125": ("hertz(S.dense_cluster(125, seed=5, velocity_sigma=0.1), memory=False)", 10, 30),
    "hertz_memory216_rolling": ("hertz(S.dense_cluster(216, seed=6, velocity_sigma=0.1), memory=True)", 10, 30),
    "loadings125": ("loaded(S.dense_cluster(125, seed=7, velocity_sigma=0.05))", 10, 18),
    "convex216_gjk_sv": ("signed_volumes(S.convex_box(216, seed=8, converge_time=0.004, velocity_sigma=0.05))",
                         900, 5),
}


def converge(sc, target, T):
    """Adds a velocity field that brings every particle to `target` in time T:
    a dense cluster against the drum's rotating shell after about T."""
    sc.particles["velocity"] = sc.particles["velocity"] + (np.asarray(target) - sc.particles["position"]) / T
    return sc


def rolling(sc):
    laws = []
    for a, b, law, prm in sc.laws[0]:
        prm = list(prm)
        prm[5] = 0.05   # mur
        prm[6] = 0.3    # etarpf
        laws.append((a, b, law, prm))
    sc.laws = [laws]
    return sc


def hooke(sc):
    from pacific_b200.abi import HOOKE
    sc.laws = [[(a, b, HOOKE, [prm[0], prm[1], prm[2], prm[3], 1.0e-3]) for a, b, law, prm in sc.laws[0]]]
    return sc


def hertz(sc, memory):
    """Hertz (Es = 1 GPa, Gs = 0.3 GPa, en = 0.8, muc = 0.4, kr = 1e-3) or
    HertzMemory (same moduli, mur = 0.05, etarpf = 0.3) on every pair;
    dt = 2e-6 s, a twentieth of the Hertz contact time at 0.1 m/s."""
    from pacific_b200.abi import HERTZ, HERTZ_MEMORY
    Es, Gs = 1.0e9, 0.3e9
    if memory:
        sc.laws = [[(a, b, HERTZ_MEMORY, [Es, 0.8, 0.4, Gs, 0.05, 0.3, 0.0]) for a, b, law, prm in sc.laws[0]]]
    else:
        sc.laws = [[(a, b, HERTZ, [Es, 0.8, 0.4, 1.0e-3, Gs]) for a, b, law, prm in sc.laws[0]]]
    sc.dt = 2.0e-6
    return sc


def loaded(sc):
    """Imposed motions of every kind on the six walls (ids -1..-6 = x, X, y, Y,
    z, Z), with time windows that open and close during the replayed steps
    (t = 1e-4 .. 2.8e-4 s): a sinusoidal floor, a crenel on x [1e-4, 3e-4], a
    multi-sinusoid on y, a translation plus a rotation about its own centre
    starting at 2e-4 on the top, a rotation about the box centre on X
    [5e-5, 2.5e-4], and a translation on Y that ends at 2e-4."""
    from pacific_b200.abi import (CONSTANT_ROTATION, CONSTANT_TRANSLATION, CRENEL_TRANSLATION,
                                  MULTISIN_TRANSLATION, SIN_TRANSLATION)
    d = sc.domains[0]
    centre = list(np.asarray(d["origin"]) + np.asarray(d["size"]) / 2.0)
    sc.meta["loadings"] = [[
        dict(obstacle_id=-5, type=SIN_TRANSLATION, vector=(0, 0, 1), amplitude=0.05, period=2e-3, phase_deg=30.0),
        dict(obstacle_id=-1, type=CRENEL_TRANSLATION, t_start=1e-4, t_end=3e-4, vector=(1, 0, 0), amplitude=0.02,
             period=5e-5),
        dict(obstacle_id=-3, type=MULTISIN_TRANSLATION, vector=(1, 1, 0), amplitude=(0.01, 0.02, 0.0),
             period=(1e-3, 1.3e-3, 1.0), phase_deg=(0.0, 90.0, 0.0)),
        dict(obstacle_id=-6, type=CONSTANT_TRANSLATION, vector=(0, 0, -0.01)),
        dict(obstacle_id=-6, type=CONSTANT_ROTATION, t_start=2e-4, vector=(0, 0, 20.0)),
        dict(obstacle_id=-2, type=CONSTANT_ROTATION, t_start=5e-5, t_end=2.5e-4, vector=(0, 5.0, 0), center=centre),
        dict(obstacle_id=-4, type=CONSTANT_TRANSLATION, t_end=2e-4, vector=(0, -0.02, 0)),
    ]]
    for o in sc.obstacles[0]:
        o["moving"] = 1
    return sc


def signed_volumes(sc):
    """The signed-volume GJK (<CollisionDetection Type="GJK_SV"/>) for the
    pairs of non-spherical bodies."""
    from pacific_b200.abi import GJK_SV
    sc.meta["collision"] = GJK_SV
    return sc


def warm_case(name):
    """First process: the reference advances the scenario `warm` steps; its
    state and contact memory become the fixture's input."""
    from pacific_b200 import scenarios as S  # noqa: F401
    from pacific_b200.abi import FP64, GrainsLib, Simulation
    import golden_io as G
    expr, warm, steps = CASES[name]
    sc = eval(expr)
    lib = GrainsLib(REF_SO, "grains_ref_")
    sim = Simulation(lib, FP64, max_particles=sc.n)
    S.apply(sim, sc)
    sim.initialize_leapfrog(0.0, sc.dt)
    t = sim.step(warm, 0.0, sc.dt) if warm else 0.0
    st = sim.download()
    mem = sim.contact_memory()
    for k in G.STATE_KEYS:
        sc.particles[k] = st[k]
    if any(sc.shapes[k][0] != S.SPHERE for k in set(np.asarray(sc.particles["shape"]).tolist())):
        sc.particles["basis"] = st["basis"]
    out = G.scenario_to_npz_dict(sc)
    out.update(G.memory_arrays(mem, "mem_in_"))
    out["time"] = np.array(t)
    out["after_steps"] = np.array(steps)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def replay_case(name):
    """Second process: a fresh reference context is given the recorded input,
    exactly as the tests give it to the oracle and the CUDA path, and its
    results become the fixture's expected output.  (A fresh context matters:
    the reference's cell lists keep an order that depends on the history, so
    the order of the force sums, and hence their last bits, differs between a
    continuing run and a replay.)"""
    from pacific_b200 import scenarios as S  # noqa: F401
    from pacific_b200.abi import FP64, GrainsLib, Simulation
    import golden_io as G
    path = os.path.join(HERE, name + ".npz")
    z = np.load(path)
    out = {k: z[k] for k in z.files}
    sc = G.scenario_from_npz(z)
    lib = GrainsLib(REF_SO, "grains_ref_")
    sim = Simulation(lib, FP64, max_particles=sc.n)
    S.apply(sim, sc)
    sim.upload_contact_memory(G.memory_from(z, "mem_in_"))
    t = float(z["time"])
    sim.compute_forces(t, sc.dt)
    d = sim.download()
    out["force"] = d["force"]
    out["torque"] = d["torque"]
    out["coordination"] = d["coordination"]
    # contact pairs are read from the reference's contact-memory maps, which
    # only the memory laws (HookeMemory, HertzMemory) fill
    out["has_contact_pairs"] = np.array(all(l[2] in (1, 3) for l in sc.laws[0]))
    out["contact_pairs"] = sim.contact_pairs()
    out["candidate_pairs"] = sim.candidate_pairs()
    out.update(G.memory_arrays(sim.contact_memory(), "mem_out_"))
    steps = int(z["after_steps"])
    sim.step(steps, t, sc.dt)
    d = sim.download()
    for k in G.STATE_KEYS + ["force", "torque"]:
        out["after_" + k] = d[k]
    if "in_basis" in out:
        out["after_basis"] = d["basis"]
    out.update(G.memory_arrays(sim.contact_memory(), "mem_after_"))
    if sc.meta.get("loadings"):
        out["after_obstacles"] = sim.obstacles(0, len(sc.obstacles[0]))
    np.savez_compressed(path, **out)
    print("%s: %d particles, %d contacts, %d candidates" % (name, sc.n, len(out["contact_pairs"]),
                                                           len(out["candidate_pairs"])))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] in ("--warm", "--replay"):
        (warm_case if sys.argv[1] == "--warm" else replay_case)(sys.argv[2])
        sys.exit(0)
    if not os.path.exists(REF_SO):
        sys.exit("build the reference first: make -C oracle/ref")
    for name in (sys.argv[1:] or CASES):
        subprocess.run([sys.executable, __file__, "--warm", name], check=True)
        subprocess.run([sys.executable, __file__, "--replay", name], check=True)
