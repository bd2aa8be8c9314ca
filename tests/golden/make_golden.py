#!/usr/bin/env python
"""Generates the golden fixtures of tests/golden/*.npz by running the
reference Grains3D itself (oracle/_ref/libgrains_ref.so, built from the
reference sources by oracle/ref/Makefile) on seeded scenarios.

Each case: the reference advances a scenario for `warm` steps (building up
contact memory), its state and memory are recorded as the input, then one
force evaluation (forces, torques, coordination, contact and candidate pairs,
memory) and `steps` further KDK steps (positions, velocities, quaternions,
angular velocities) are recorded as the expected output.  Every case runs in
its own process because the reference keeps process-wide static state.

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
}


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


def run_case(name):
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
    out = G.scenario_to_npz_dict(sc)
    out.update(G.memory_arrays(mem, "mem_in_"))
    out["time"] = np.array(t)
    sim.compute_forces(t, sc.dt)
    d = sim.download()
    out["force"] = d["force"]
    out["torque"] = d["torque"]
    out["coordination"] = d["coordination"]
    # contact pairs are read from the reference's contact-memory maps, which
    # only the HookeMemory law fills
    out["has_contact_pairs"] = np.array(all(l[2] == 1 for l in sc.laws[0]))
    out["contact_pairs"] = sim.contact_pairs()
    out["candidate_pairs"] = sim.candidate_pairs()
    out.update(G.memory_arrays(sim.contact_memory(), "mem_out_"))
    t2 = sim.step(steps, t, sc.dt)
    d = sim.download()
    for k in G.STATE_KEYS + ["force", "torque"]:
        out["after_" + k] = d[k]
    out["after_steps"] = np.array(steps)
    out.update(G.memory_arrays(sim.contact_memory(), "mem_after_"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("%s: %d particles, %d contacts, %d candidates" % (name, sc.n, len(out["contact_pairs"]),
                                                           len(out["candidate_pairs"])))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--case":
        run_case(sys.argv[2])
        sys.exit(0)
    if not os.path.exists(REF_SO):
        sys.exit("build the reference first: make -C oracle/ref")
    for name in (sys.argv[1:] or CASES):
        subprocess.run([sys.executable, __file__, "--case", name], check=True)
