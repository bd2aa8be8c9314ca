"""Force-driven obstacles on the CUDA path against the oracle (which
tests/test_force_obstacle_cpu.py holds to the reference): the lid of the
pressed box under an imposed force of 0.05 N, in 50-step calls (CUDA graphs
of 16 steps and the uncaptured remainder).  The contact force on the lid is
summed on the device in another order than the oracle's (a fixed tree over
fixed blocks).  FP64, 300 steps: lid within 1e-13 m and particles within
1e-12 m of the oracle (measured on B200: equal).  Mixed precision (contact
forces in FP32), 150 steps, before the impact on the bed amplifies the FP32
rounding: lid within 1e-9 m (measured 8.9e-11 m), particles within 5e-6 m
(measured 7.8e-7 m).  The convex case (64 cubes, cylinders and octahedra,
dt = 2 us, the oracle with the CUDA path's polyhedron support rule): FP64,
1,200 steps, lid within 1e-13 m and bodies within 1e-12 m (measured: equal);
mixed, 1,000 steps, lid within 1e-8 m (measured 1.8e-9 m), bodies within
1e-7 m (measured 2.0e-8 m)."""
import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED

from helpers import make

pytestmark = pytest.mark.gpu
LID = 5


def run(lib, sc, precision=None, steps=300, every=50):
    s = make(lib, sc, precision) if precision is not None else make(lib, sc)
    if precision is None:
        s.set_polyhedron_support(2)  # the oracle with the CUDA path's hill-climb start
    s.initialize_leapfrog(0.0, sc.dt)
    t, lid = 0.0, []
    for _ in range(steps // every):
        t = s.step(every, t, sc.dt)
        lid.append(s.obstacles(0, 6)[LID].copy())
    d = s.download()
    assert s.stats()["status"] == 0
    s.close()
    return np.array(lid), d


BARS = {  # (steps, lid bar, particle bar)
    ("spheres", FP64): (300, 1e-13, 1e-12),
    ("spheres", MIXED): (150, 1e-9, 5e-6),
    ("convex", FP64): (1200, 1e-13, 1e-12),
    ("convex", MIXED): (1000, 1e-8, 1e-7),
}


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("case", ["spheres", "convex"])
def test_force_driven_lid_follows_the_oracle(oracle_lib, gpu_lib, case, precision):
    sc = S.pressed_box(64, seed=4, convex=True) if case == "convex" else S.pressed_box()
    steps, tol_lid, tol_pos = BARS[(case, precision)]
    lo, do = run(oracle_lib, sc, steps=steps)
    lg, dg = run(gpu_lib, sc, precision, steps=steps)
    assert np.max(np.abs(lg[:, 9:] - lo[:, 9:])) < tol_lid
    assert np.max(np.abs(dg["position"] - do["position"])) < tol_pos
    assert np.ptp(lg[:, 11]) > 1e-4  # the lid went down to the bed and the controller moved it


def test_persistent_request_runs_the_launched_steps(gpu_lib):
    """The persistent launch does not run imposed forces: a context with a
    force-driven obstacle that asks for it runs the launched steps, to the
    same bits."""
    sc = S.pressed_box()
    runs = []
    for persistent in (0, 1):
        s = make(gpu_lib, sc, FP64)
        s.set_tuning(persistent=persistent)
        s.initialize_leapfrog(0.0, sc.dt)
        t = s.step(37, 0.0, sc.dt)
        s.step(26, t, sc.dt)
        d = s.download()
        d["lid"] = s.obstacles(0, 6)[LID].copy()
        assert s.stats()["status"] == 0
        runs.append(d)
        s.close()
    for k in ["position", "velocity", "lid"]:
        assert np.array_equal(runs[0][k], runs[1][k]), k
