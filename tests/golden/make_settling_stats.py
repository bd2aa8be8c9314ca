#!/usr/bin/env python
"""Generates tests/golden/settling_1k_stats.npz: the run statistics of the
config-0 settling case (1,000 spheres r = 1 mm dropped in a closed 20x20x60 mm
box, HookeMemory kn = 1e5, en = 0.9, mu = 0.5, kt = 0.8 kn, dt = 1e-5 s) computed
by the reference Grains3D itself (oracle/_ref/libgrains_ref.so, built from the
reference sources by oracle/ref/Makefile) over 30,000 steps: the 10,000 steps
of the configuration and 20,000 more in which the bed comes to rest.

Recorded every 500 steps: kinetic energy, mean height and mean coordination
number (Particle::getCoordinationNumber, Particle.cpp:1703-1707).  At the end:
the packing fraction of the bed in the slab between 20 % and 70 % of its
height, and the run statistics of AppCollision::addToContactsFeatures
(AppCollision.cpp:160-187) over the whole run: the largest overlap and the
mean overlap of every contact met.

    python tests/golden/make_settling_stats.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")
STEPS, EVERY = 30000, 500


def packing_fraction(position, radius, lx, ly):
    """Solid fraction of the slab [0.2 h, 0.7 h] of the bed (h: the 95th
    percentile of the centres' heights plus a radius), from the sphere
    centres inside it: each counts its whole volume."""
    z = position[:, 2]
    h = float(np.quantile(z, 0.95)) + float(np.max(radius))
    lo, hi = 0.2 * h, 0.7 * h
    inside = (z >= lo) & (z < hi)
    vol = float(np.sum(4.0 / 3.0 * np.pi * radius[inside] ** 3))
    return vol / (lx * ly * (hi - lo))


def run(lib, sc, precision=None, steps=STEPS, every=EVERY):
    """The statistics of a run of `sc` on the implementation `lib`: the
    history (every `every` steps: step, kinetic energy, mean height, mean
    coordination), the packing fraction at the end, and the running overlap
    maximum and mean of the whole run."""
    from pacific_b200.abi import FP64, Simulation
    from pacific_b200 import scenarios as S
    sim = Simulation(lib, FP64 if precision is None else precision, max_particles=sc.n)
    try:
        S.apply(sim, sc)
        m = np.asarray(sc.particles["mass"])
        rows = []
        sim.reset_stats()
        sim.initialize_leapfrog(0.0, sc.dt)
        t = 0.0
        for k in range(steps // every):
            t = sim.step(every, t, sc.dt)
            d = sim.download()
            ke = 0.5 * float(np.sum(m * np.sum(d["velocity"] ** 2, axis=1)))
            rows.append([(k + 1) * every, ke, float(d["position"][:, 2].mean()), float(d["coordination"].mean())])
        st = sim.stats()
        dom = sc.domains[0]
        phi = packing_fraction(d["position"], np.asarray(sc.particles["radius"]), dom["size"][0], dom["size"][1])
        return np.asarray(rows), phi, st["overlap_max"], st["overlap_mean"]
    finally:
        sim.close()


def main():
    from pacific_b200 import scenarios as S
    from pacific_b200.abi import GrainsLib
    lib = GrainsLib(REF_SO, "grains_ref_")
    rows, phi, omax, omean = run(lib, S.settling_1k())
    np.savez_compressed(os.path.join(HERE, "settling_1k_stats.npz"), history=rows, packing_fraction=phi,
                        overlap_max=omax, overlap_mean=omean,
                        columns=np.array(["step", "kinetic_energy", "mean_z", "mean_coordination"]))
    print("packing fraction %.4f, final coordination %.3f, KE %.3g, overlap max %.3g mean %.3g" %
          (phi, rows[-1, 3], rows[-1, 1], omax, omean))


if __name__ == "__main__":
    main()
