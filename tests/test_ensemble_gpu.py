"""Several independent systems in one context -- the batched path of the
ensemble workload -- against one oracle run per system.

Reference: Grains::computeParticlesForceAndTorque (Base/src/Grains.cpp:459-482)
and the KDK loop run each system on its own; the device runs every system in
the same launches, with per-system cell, law and obstacle offsets, per-system
particle ids (every system numbers its particles from 0 here, so the contact
memory must tell systems apart by row, not by id) and moving obstacles in one
of them.  The systems differ in size, in the contact-law parameters, in their
obstacle sets and in the law itself (HookeMemory, Hooke).

Bars: contact pairs, candidate pairs and coordination numbers exact; plain
FP64 forces within 1e-12 of the oracle (floor: the particle weight),
positions within 1e-13 m after 20 steps, obstacle poses within 1e-14 m; mixed
precision per-contact forces within 1e-5 (the north star's contact-force bar)
on the first force evaluation."""
import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import CONSTANT_TRANSLATION, CRENEL_TRANSLATION, FP64, HOOKE, MIXED

from helpers import make, pair_set, rel_err

pytestmark = pytest.mark.gpu


def three_systems():
    a = S.dense_cluster(125, seed=21, velocity_sigma=0.1)
    b = S.small_box(216, seed=22, velocity_sigma=0.3)
    c = S.dense_cluster(64, seed=23, velocity_sigma=0.05)
    kn_b, kn_c = 1.3e5, 6.0e4
    b.laws = [[(m0, m1, S.HOOKE_MEMORY, S.hooke_memory_params(kn_b, 0.6, 0.3, 0.8 * kn_b)) for m0, m1, _, _ in
               b.laws[0]]]
    c.laws = [[(m0, m1, HOOKE, [kn_c, 0.8, -1.0, 0.7, 0.0]) for m0, m1, _, _ in c.laws[0]]]
    b.obstacles = [[o for o in b.obstacles[0] if o["id"] != -6]]  # no top wall
    for o in c.obstacles[0]:
        o["moving"] = 1
    # imposed motions without trigonometry, so that the walls' poses are the
    # oracle's bit for bit
    c.meta["loadings"] = [[dict(obstacle_id=-5, type=CRENEL_TRANSLATION, vector=(0, 0, 1), amplitude=0.05,
                                period=6e-5),
                           dict(obstacle_id=-6, type=CONSTANT_TRANSLATION, vector=(0, 0, -0.02))]]
    return [a, b, c]


def merge(scs):
    """One scenario holding every system of `scs` (same dt)."""
    shapes, parts, doms, laws, obstacles, loads = [], [], [], [], [], []
    for s, sc in enumerate(scs):
        off = len(shapes)
        shapes += sc.shapes
        p = dict(sc.particles)
        p["shape"] = np.asarray(p["shape"]) + off
        p["system"] = np.full(sc.n, s, np.int32)
        parts.append(p)
        doms += sc.domains
        laws += sc.laws
        obstacles.append([dict(o, shape=o["shape"] + off) for o in sc.obstacles[0]])
        loads.append((sc.meta.get("loadings") or [[]])[0])
    keys = parts[0].keys()
    p = {k: (np.concatenate([q[k] for q in parts]) if parts[0][k] is not None else None) for k in keys}
    return S.Scenario("three_systems", shapes, doms, laws, obstacles, p, scs[0].dt, 20, meta=dict(loadings=loads))


def split(arr, scs, s):
    lo = sum(sc.n for sc in scs[:s])
    return arr[lo:lo + scs[s].n]


def weight(sc):
    return float(np.min(sc.particles["mass"])) * 9.81


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_systems_in_one_context_match_separate_oracle_runs(oracle_lib, gpu_lib, precision):
    scs = three_systems()
    sim = make(gpu_lib, merge(scs), precision)
    oracles = [make(oracle_lib, sc) for sc in scs]
    # the first force evaluation (empty contact memory)
    sim.compute_forces(0.0, scs[0].dt)
    d = sim.download()
    assert int(d["coordination"].sum()) > 500
    for s, (sc, o) in enumerate(zip(scs, oracles)):
        o.compute_forces(0.0, sc.dt)
        do = o.download()
        assert np.array_equal(split(d["coordination"], scs, s), do["coordination"]), s
        assert pair_set(sim.contact_pairs(s)) == pair_set(o.contact_pairs()), s
        assert np.array_equal(sim.candidate_pairs(s), o.candidate_pairs()), s
        pg, fg = sim.contact_forces(s)
        po, fo = o.contact_forces()
        assert np.array_equal(pg, po)
        if precision == FP64:
            assert rel_err(split(d["force"], scs, s), do["force"], weight(sc)) < 1e-12, s
            assert rel_err(fg, fo, weight(sc)) < 1e-12, s
        else:
            assert rel_err(fg, fo, weight(sc)) < 1e-5, s
    if precision == MIXED:
        return
    # 20 KDK steps: the contact memory of every system, the moving walls
    sim.initialize_leapfrog(0.0, scs[0].dt)
    t = sim.step(20, 0.0, scs[0].dt)
    d = sim.download()
    states, mems = [], []
    for s, (sc, o) in enumerate(zip(scs, oracles)):
        o.initialize_leapfrog(0.0, sc.dt)
        to = o.step(20, 0.0, sc.dt)
        assert to == pytest.approx(t)
        do = o.download()
        assert np.max(np.abs(split(d["position"], scs, s) - do["position"])) < 1e-13, s
        n_obs = len(sc.obstacles[0])
        assert np.array_equal(sim.obstacles(s, n_obs), o.obstacles(0, n_obs)), s
        states.append(do)
        m = o.contact_memory()
        m["system"] = np.full(len(m["owner"]), s, np.int32)
        mems.append(m)
    # the next force evaluation from the oracles' states and contact memories
    # (uploaded with their systems: the ids repeat across systems)
    sim.update({k: np.concatenate([st[k] for st in states]) for k in ["position", "quaternion", "velocity", "omega"]})
    sim.upload_contact_memory({k: np.concatenate([m[k] for m in mems]) for k in mems[0]})
    sim.compute_forces(t, scs[0].dt)
    d = sim.download()
    for s, (sc, o) in enumerate(zip(scs, oracles)):
        o.compute_forces(t, sc.dt)
        do = o.download()
        assert np.array_equal(split(d["coordination"], scs, s), do["coordination"]), s
        assert int(do["coordination"].sum()) > 20, s
        assert pair_set(sim.contact_pairs(s)) == pair_set(o.contact_pairs()), s
        assert rel_err(split(d["force"], scs, s), do["force"], weight(sc)) < 1e-12, s
        assert rel_err(split(d["torque"], scs, s), do["torque"], weight(sc) * 1e-3) < 1e-10, s
