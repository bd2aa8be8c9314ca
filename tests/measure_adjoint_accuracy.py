"""Measures the adjoint's gradients on the full adjoint workload (4,096
spheres, a checkpoint every 100 force evaluations) against the FP64
dual-number oracle (oracle/tangent_oracle.cpp), at several horizons up to the
full 2,000 steps, in both precisions, and prints one JSON line.  Run on a GPU
machine:  python tests/measure_adjoint_accuracy.py

Directions: one per law parameter (kn, en, muc, kt; both laws) and two unit
random directions of the initial velocities.  Beyond the first collisions the
dynamics is chaotic, so the derivatives themselves grow by orders of magnitude
and the agreement measures how far two exact derivative computations of the
same discrete map (reverse mode on the GPU, forward mode on the CPU) stay
together under rounding."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import pacific_b200  # noqa: E402
from pacific_b200 import scenarios as S  # noqa: E402
from pacific_b200.abi import FP64, MIXED, Adjoint  # noqa: E402

from helpers import make, tangent_run  # noqa: E402


def main(horizons=(100, 200, 500, 2000)):
    lib = pacific_b200.load_library()
    sc = S.adjoint_4k()
    n = sc.n

    def loss_grads(final):
        m = sc.particles["mass"]
        inertia = np.asarray(sc.particles["inertia"])[:, 0]
        v, w = final["velocity"], final["omega"]
        zc = final["position"][:, 2].mean()
        ke = np.mean(0.5 * m * (v * v).sum(1) + 0.5 * inertia * (w * w).sum(1))
        gx = np.zeros_like(v)
        gx[:, 2] = 2.0 * 0.1 * zc / n
        return gx, 2.0 * 0.5 * ke * (m[:, None] * v) / n, 2.0 * 0.5 * ke * (inertia[:, None] * w) / n

    rng = np.random.default_rng(9)
    nd = 6
    dv = np.zeros((nd, n, 3))
    dl = np.zeros((nd, 16, 4))
    for t in range(4):
        dl[t, [0, 1, 4], t] = 1.0
    for t in range(4, nd):
        d = rng.normal(size=(n, 3))
        dv[t] = d / np.linalg.norm(d)
    out = {}
    for horizon in horizons:
        ofin, tan = tangent_run(sc, horizon, dv, dl)
        gx, gv, gw = loss_grads(ofin)
        dual = np.array([(gx * tan["position"][k]).sum() + (gv * tan["velocity"][k]).sum() +
                         (gw * tan["omega"][k]).sum() for k in range(nd)])
        row = {"dual": dual.tolist()}
        for name, prec in [("fp64", FP64), ("mixed", MIXED)]:
            sim = make(lib, sc, prec)
            adj = Adjoint(sim, 100)
            fin = adj.forward(horizon, sc.dt)
            g = adj.backward(*loss_grads(fin))
            ad = np.array([(g["velocity"] * dv[k]).sum() + (g["laws"] * dl[k]).sum() for k in range(nd)])
            rel = np.abs(ad - dual) / np.abs(dual)
            row[name] = {"max_rel": float(rel.max()), "median_rel": float(np.median(rel)), "adjoint": ad.tolist(),
                         "contacts": adj.signature()[1]}
            adj.close()
            sim.close()
        out[str(horizon)] = row
    print(json.dumps({"workload": "adjoint_4k", "directions": "kn, en, muc, kt, 2 random unit velocity directions",
                      "horizons": out}))


if __name__ == "__main__":
    main()
