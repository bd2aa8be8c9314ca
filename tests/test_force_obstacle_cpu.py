"""Force-driven obstacles (ObstacleImposedForce "ConstantTranslation",
Component/src/ObstacleImposedForce.cpp:183-252, driven by
ObstacleKinematicsForce::ImposedMotion and SimpleObstacle::Move): the oracle
against the reference itself (oracle/_ref), which reads the same loading from
its XML input (<ObstacleLoading Type="Force">, Base/src/Grains.cpp:1719-1745).
A lid lowered onto a bed of 125 spheres with an imposed force of 0.05 N: it
moves down at Vmax until the spheres push back, then the PID controller drives
the contact force on it towards the imposed force.  Over the first 300 steps
(the lid's approach, the impact, its rebound and the controller's
corrections) the lid's pose and the particle positions are equal to the bit;
the particle velocities differ by one unit in the last place, as the oracle's
and the reference's sphere runs do without any loading (1.4e-17 m/s, angular
velocities 1.1e-14 rad/s).  Skipped where the reference library is not
built."""
import os
import subprocess
import sys

import numpy as np
import pytest

from pacific_b200 import scenarios as S

from helpers import make

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")
LID = 5  # index of the lid (the upper z wall) in the obstacle list


def ref_run(tmp_path, case, steps, every):
    """The reference's run of a pressed-box case in a process of its own: the
    reference keeps the imposed-force controller's history in static
    variables (ObstacleImposedForce.cpp:208-212), which carry over from one
    context to the next within a process."""
    if not os.path.exists(REF_SO):
        pytest.skip("the reference library is not built (needs the reference sources)")
    out = tmp_path / "ref.npz"
    code = (
        "import sys, numpy as np\n"
        "sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
        "from test_force_obstacle_cpu import run, case_scenario\n"
        "from pacific_b200.abi import GrainsLib\n"
        "lid, d = run(GrainsLib(%r, 'grains_ref_'), case_scenario(%r), %d, %d)\n"
        "np.savez(%r, lid=lid, position=d['position'], velocity=d['velocity'], omega=d['omega'])\n"
    ) % (ROOT, os.path.join(ROOT, "tests"), REF_SO, case, steps, every, str(out))
    subprocess.run([sys.executable, "-c", code], check=True, timeout=600)
    r = np.load(out)
    return r["lid"], {k: r[k] for k in ["position", "velocity", "omega"]}


def case_scenario(case):
    return S.pressed_box(64, seed=4, convex=True) if case == "convex" else S.pressed_box()


def run(lib, sc, steps, every):
    s = make(lib, sc)
    s.initialize_leapfrog(0.0, sc.dt)
    t, lid = 0.0, []
    for _ in range(steps // every):
        t = s.step(every, t, sc.dt)
        lid.append(s.obstacles(0, 6)[LID].copy())
    d = s.download()
    s.close()
    return np.array(lid), d


def test_force_driven_lid_matches_the_reference(oracle_lib, tmp_path):
    sc = case_scenario("spheres")
    z0 = sc.obstacles[0][LID]["transform"][11]
    la, da = ref_run(tmp_path, "spheres", 300, 10)
    lb, db = run(oracle_lib, sc, 300, 10)
    assert np.array_equal(la, lb)
    assert np.array_equal(da["position"], db["position"])
    assert np.max(np.abs(da["velocity"] - db["velocity"])) < 1e-15
    assert np.max(np.abs(da["omega"] - db["omega"])) < 1e-12
    # the lid went down, met the bed and was driven back up by the controller
    z = lb[:, 11]
    assert z[1] < z0 and np.max(z) > z[1]


def test_force_driven_lid_on_convex_bodies_matches_the_reference(oracle_lib, tmp_path):
    """64 cubes, cylinders and octahedra under the lid, 1,200 steps of 2 us
    (the lid reaches the bodies after about 150 steps and is then pressed into
    the settling bed): everything equal to the bit."""
    sc = case_scenario("convex")
    la, da = ref_run(tmp_path, "convex", 1200, 20)
    lb, db = run(oracle_lib, sc, 1200, 20)
    assert np.array_equal(la, lb)
    for k in ["position", "velocity", "omega"]:
        assert np.array_equal(da[k], db[k]), k
    assert lb[-1, 11] < lb[10, 11] - 1e-4  # pressed down after the contact


def test_imposed_force_loading_is_validated(oracle_lib):
    sc = S.pressed_box()
    s = make(oracle_lib, sc)
    with pytest.raises(Exception):
        s.set_obstacle_loadings(0, [dict(obstacle_id=-6, type=5, vector=(0.0, 0.0, 0.0), amplitude=(1e-5, 1.0))])
    s.close()
