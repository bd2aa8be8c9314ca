"""The options of the reference's <CollisionDetection> element on the CUDA path
(Base/src/Grains.cpp:654-723): the GJK tolerance, the Nesterov-accelerated
search direction (Acceleration="ON", Convex.cpp:566-597) and the warm start of
every convex pair from its last GJK iterate (History="ON", the
CollisionHistory of Particle.cpp:486-505, Convex.cpp:636-716).

From a dense cluster of cubes, cylinders and octahedra advanced by the oracle
(about 950 GJK runs per step), the oracle and the FP64 CUDA path start with
empty histories and take two steps with each option set: the same GJK calls
and iteration counts, positions at rounding level.  Further on the two drift
apart at rounding level whatever the options (the force sums run in another
order, and near-degenerate contacts amplify it: 2e-9 m after 20 steps without
any option), so the iteration counts of longer runs differ by a few in 1e5.
The CUDA path keeps a pair's history with its lower id, where the reference
keeps it with whichever particle called the interaction; the two agree while
that role does not change."""
import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, GJK, GJK_SV, MIXED

from helpers import make

pytestmark = pytest.mark.gpu

OPTIONS = [dict(history=True), dict(acceleration=True), dict(history=True, acceleration=True),
           dict(tolerance=1e-6)]


def dense_convex(oracle_lib):
    sc = S.convex_box(216, seed=7, converge_time=2e-3)
    o = make(oracle_lib, sc)
    o.set_polyhedron_support(2)
    o.initialize_leapfrog(0.0, sc.dt)
    t = o.step(450, 0.0, sc.dt)
    st = o.download()
    mem = o.contact_memory()
    o.close()
    p = dict(sc.particles)
    for k in ["position", "quaternion", "basis", "velocity", "omega"]:
        p[k] = st[k]
    sc.particles = p
    return sc, mem, t


@pytest.fixture(scope="module")
def dense(oracle_lib):
    return dense_convex(oracle_lib)


def run(lib, sc, mem, t, options, algorithm, precision=FP64, oracle=False, steps=60):
    sc.meta = dict(sc.meta or {}, collision_options=options, collision=algorithm)
    s = make(lib, sc, precision)
    if oracle:
        s.set_polyhedron_support(2)
    s.upload_contact_memory(mem)
    s.initialize_leapfrog(t, sc.dt)
    s.reset_stats()
    s.step(steps, t, sc.dt)
    d, st = s.download(), s.stats()
    s.close()
    return d, st


@pytest.mark.parametrize("algorithm", [GJK, GJK_SV], ids=["johnson", "sv"])
@pytest.mark.parametrize("options", OPTIONS, ids=["history", "accel", "history_accel", "tol1e-6"])
def test_collision_options_follow_the_oracle(oracle_lib, gpu_lib, dense, options, algorithm):
    sc, mem, t = dense
    do, so = run(oracle_lib, sc, mem, t, options, algorithm, oracle=True, steps=2)
    dg, sg = run(gpu_lib, sc, mem, t, options, algorithm, steps=2)
    assert so["n_gjk_calls"] > 1500
    assert sg["n_gjk_calls"] == so["n_gjk_calls"]
    if algorithm == GJK:
        assert sg["n_gjk_iterations"] == so["n_gjk_iterations"]
        assert np.max(np.abs(dg["position"] - do["position"])) < 1e-14
    else:
        # the signed-volume sub-algorithm is written from the paper in its own
        # arithmetic (the oracle follows the reference's), and it stops as soon
        # as a new support point drops out of the simplex, where the
        # reference's loop goes on until the optimality gap or a repeated
        # point stops it: up to 20 % fewer iterations on this cluster, distances
        # within the GJK tolerance (positions 3e-11 m apart after two steps)
        assert sg["n_gjk_iterations"] <= 1.01 * so["n_gjk_iterations"]
        assert np.max(np.abs(dg["position"] - do["position"])) < 1e-10
    assert np.array_equal(dg["coordination"], do["coordination"])


def test_warm_start_saves_gjk_iterations(gpu_lib, dense):
    """The history's purpose: fewer GJK iterations per call on the same run
    (the reference: 8.70 instead of 9.76 per call on this cluster)."""
    sc, mem, t = dense
    _, cold = run(gpu_lib, sc, mem, t, dict(history=False), GJK)
    _, warm = run(gpu_lib, sc, mem, t, dict(history=True), GJK)
    mean = lambda s: s["n_gjk_iterations"] / s["n_gjk_calls"]
    assert mean(warm) < 0.95 * mean(cold)


def test_history_in_mixed_precision(gpu_lib, dense):
    """The mixed-precision path with the warm start: GJK runs in double in
    both precisions, so the same GJK calls, and positions within the mixed
    bar of the golden tests (2e-7 m; FP32 force rounding amplified by the
    dense packing: 1.3e-8 m measured after 5 steps) of the FP64 run."""
    sc, mem, t = dense
    d64, s64 = run(gpu_lib, sc, mem, t, dict(history=True), GJK, steps=5)
    dm, sm = run(gpu_lib, sc, mem, t, dict(history=True), GJK, precision=MIXED, steps=5)
    assert sm["n_gjk_calls"] == s64["n_gjk_calls"]
    assert np.max(np.abs(dm["position"] - d64["position"])) < 2e-7


def test_options_on_spheres(gpu_lib):
    """Sphere pairs never run GJK: the options leave a sphere run unchanged."""
    sc = S.small_box(125, seed=7)
    a = make(gpu_lib, sc, FP64)
    sc.meta = dict(sc.meta or {}, collision_options=dict(history=True, acceleration=True))
    b = make(gpu_lib, sc, FP64)
    for s in (a, b):
        s.initialize_leapfrog(0.0, sc.dt)
        s.step(50, 0.0, sc.dt)
    assert np.array_equal(a.download()["position"], b.download()["position"])
