#!/usr/bin/env python
"""Generates tests/golden/io_*.npz: files written by the reference Grains3D
itself (oracle/_ref/libgrains_ref.so, built from the reference sources by
oracle/ref/Makefile) for the reload-file and RawData writers.

For each case the reference advances a seeded scenario `warm` steps, then
writes with its own code:

* the particle file of a reload, text and hybrid binary (AllComponents::write);
* two RawData outputs of that state, text and binary
  (RawDataPostProcessingWriter): one that starts the files, one appended at a
  later time.

The fixture holds the scenario, the exact bytes of every file, and per
particle of the files (in file order) the static data the state upload needs
(shape, material, radius, crust, mass, inertia), matched to the uploaded
particles by their exact positions.

    python tests/golden/make_io_golden.py            # all cases
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")

CASES = {
    # name: (scenario expression, warm steps)
    "io_spheres64": ("rolling(S.dense_cluster(64, seed=3, velocity_sigma=0.1))", 12),
    "io_convex27": ("S.convex_box(27, seed=4, converge_time=0.004, velocity_sigma=0.05)", 700),
}
RAW_FILES = ["_position_x.dat", "_position_y.dat", "_position_z.dat", "_translational_velocity_x.dat",
             "_translational_velocity_y.dat", "_translational_velocity_z.dat", "_angular_velocity_x.dat",
             "_angular_velocity_y.dat", "_angular_velocity_z.dat", "_coordinationNumber.dat", "_particleType.dat"]
LATER = 1.25e-3  # the appended RawData output is stamped this much later


def rolling(sc):
    laws = []
    for a, b, law, prm in sc.laws[0]:
        prm = list(prm)
        prm[5] = 0.05   # mur
        prm[6] = 0.3    # etarpf
        laws.append((a, b, law, prm))
    sc.laws = [laws]
    return sc


def run_case(name, out_dir):
    from pacific_b200 import scenarios as S  # noqa: F401
    from pacific_b200.abi import FP64, GrainsLib, Simulation
    import golden_io as G
    expr, warm = CASES[name]
    sc = eval(expr)
    lib = GrainsLib(REF_SO, "grains_ref_")
    sim = Simulation(lib, FP64, max_particles=sc.n)
    S.apply(sim, sc)
    sim.initialize_leapfrog(0.0, sc.dt)
    t = sim.step(warm, 0.0, sc.dt)
    out = {}
    for binary, key in [(False, "reload_text"), (True, "reload_bin")]:
        path = os.path.join(out_dir, key)
        sim.write_reload_particles(path, binary=binary)
        out[key] = np.frombuffer(open(path, "rb").read(), np.uint8)
    for binary, key in [(False, "raw_text"), (True, "raw_bin")]:
        root = os.path.join(out_dir, key)
        sim.write_rawdata(root, t, binary=binary, truncate=True)
        sim.write_rawdata(root, t + LATER, binary=binary, truncate=False)
        for f in RAW_FILES:
            out[key + f] = np.frombuffer(open(root + f, "rb").read(), np.uint8)
    # static data per particle of the files, matched by exact position
    st = sim.download()
    text = bytes(out["reload_text"]).decode()
    pos = [tuple(float(x) for x in line.split()[4:7]) for line in text.splitlines() if line.strip()]
    where = {tuple(p): i for i, p in enumerate(st["position"].tolist())}
    idx = np.array([where[p] for p in pos])
    p = sc.particles
    out["static_shape"] = np.asarray(p["shape"], np.int32)[idx]
    out["static_material"] = np.asarray(p["material"], np.int32)[idx]
    for k in ["radius", "crust", "mass"]:
        out["static_" + k] = np.asarray(p[k], np.float64)[idx]
    out["static_inertia"] = np.asarray(p["inertia"], np.float64)[idx]
    spec = G.scenario_to_npz_dict(sc)["spec"]
    out["spec"] = spec
    out["time"] = np.array(t)
    out["later"] = np.array(t + LATER)
    out["n_total"] = np.array(sc.n)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    spec = json.loads(str(spec))
    print("%s: %d particles, reload %d bytes (text), %d (binary)" % (name, sc.n, len(out["reload_text"]),
                                                                    len(out["reload_bin"])))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--case":
        with tempfile.TemporaryDirectory(prefix="gg_io_") as d:
            run_case(sys.argv[2], d)
        sys.exit(0)
    if not os.path.exists(REF_SO):
        sys.exit("build the reference first: make -C oracle/ref")
    for name in (sys.argv[1:] or CASES):
        # one process per case: the reference keeps process-wide static state
        subprocess.run([sys.executable, __file__, "--case", name], check=True)
