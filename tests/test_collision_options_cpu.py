"""The oracle's restatement of the <CollisionDetection> options (tolerance,
Nesterov acceleration, collision-history warm start; Base/src/Grains.cpp:
654-723, Convex.cpp:536-716, Particle.cpp:486-505) against the reference
itself (oracle/_ref, built from the reference's sources): a converging cluster
of 216 cubes, cylinders and octahedra, 200 steps, positions bit for bit with
every option set and both GJK algorithms.  Skipped where the reference library
is not built."""
import os

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import GJK, GJK_SV, GrainsLib

from helpers import make

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")
OPTIONS = [dict(history=True), dict(acceleration=True), dict(history=True, acceleration=True),
           dict(tolerance=1e-6)]


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(REF_SO):
        pytest.skip("the reference library is not built (needs the reference sources)")
    return GrainsLib(REF_SO, "grains_ref_")


def positions(lib, sc, steps=(100, 200)):
    s = make(lib, sc)
    s.initialize_leapfrog(0.0, sc.dt)
    out, t, done = [], 0.0, 0
    for n in steps:
        t = s.step(n - done, t, sc.dt)
        done = n
        out.append(s.download()["position"])
    s.close()
    return out


@pytest.mark.parametrize("algorithm", [GJK, GJK_SV], ids=["johnson", "sv"])
@pytest.mark.parametrize("options", OPTIONS, ids=["history", "accel", "history_accel", "tol1e-6"])
def test_options_match_the_reference(oracle_lib, ref_lib, options, algorithm):
    sc = S.convex_box(216, seed=7, converge_time=2e-3)
    # the options go in before the upload: the reference reads them from the
    # input file written there
    sc.meta = dict(sc.meta or {}, collision_options=options, collision=algorithm)
    for a, b in zip(positions(ref_lib, sc), positions(oracle_lib, sc)):
        assert np.array_equal(a, b)


def test_options_are_validated(oracle_lib):
    sc = S.convex_box(27, seed=7)
    s = make(oracle_lib, sc)
    with pytest.raises(Exception):
        s.set_collision_options(tolerance=1e-12)
    s.close()
