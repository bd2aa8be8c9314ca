"""Launch and grid tuning (grains_gpu_set_tuning, grains_gpu_autotune): no
tuning changes contacts or forces beyond the order of floating-point sums, and
the autotuner restores the state it started from exactly."""
import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED

from helpers import make, pair_set, rel_err

pytestmark = pytest.mark.gpu


def evolved_box():
    sc = S.small_box(343, seed=4, velocity_sigma=0.2)
    return sc


@pytest.mark.parametrize("tuning", [dict(cell_factor=1.5), dict(contacts_block=128, forces_block=64),
                                    dict(list_capacity=16), dict(gather_every=1), dict(gather_every=7)])
def test_tuning_keeps_the_physics(gpu_lib, tuning):
    sc = evolved_box()
    a, b = make(gpu_lib, sc, FP64), make(gpu_lib, sc, FP64)
    b.set_tuning(**{**dict(cell_factor=1.0, contacts_block=256, forces_block=128, list_capacity=0, gather_every=16),
                    **tuning})
    for s in (a, b):
        s.initialize_leapfrog(0.0, sc.dt)
        s.step(50, 0.0, sc.dt)
        s.compute_forces(50 * sc.dt, sc.dt)
    da, db = a.download(), b.download()
    assert pair_set(a.contact_pairs()) == pair_set(b.contact_pairs())
    weight = sc.particles["mass"][0] * 9.81
    assert rel_err(db["force"], da["force"], weight) < 1e-9
    assert np.max(np.abs(db["position"] - da["position"])) < 1e-12


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_autotune_restores_the_state(gpu_lib, precision):
    sc = evolved_box()
    sim = make(gpu_lib, sc, precision)
    sim.initialize_leapfrog(0.0, sc.dt)
    t = sim.step(20, 0.0, sc.dt)
    before, mem_before = sim.download(), sim.contact_memory()
    best, ms = sim.autotune(t, sc.dt, trial_steps=20)
    after, mem_after = sim.download(), sim.contact_memory()
    for k in ["position", "quaternion", "velocity", "omega"]:
        assert np.array_equal(before[k], after[k]), k
    assert set(zip(mem_before["owner"], mem_before["other"])) == set(zip(mem_after["owner"], mem_after["other"]))
    assert ms > 0 and best["cell_factor"] >= 1.0 and sim.tuning() == best
    sim.step(10, t, sc.dt)   # the tuned context keeps running


def test_gather_period_gives_identical_runs(gpu_lib):
    """The particle arrays permuted into cell order every step or every 5th
    step (between, the cell lists are reached through the permutation): the
    same sums in the same order, hence identical bits, through graphs and the
    uncaptured remainder steps alike."""
    sc = evolved_box()
    runs = []
    for ge in (1, 5):
        s = make(gpu_lib, sc, FP64)
        s.set_tuning(gather_every=ge)
        s.initialize_leapfrog(0.0, sc.dt)
        t = s.step(37, 0.0, sc.dt)
        s.step(26, t, sc.dt)
        runs.append(s.download())
        s.close()
    for k in ["position", "velocity", "omega", "force"]:
        assert np.array_equal(runs[0][k], runs[1][k]), k


def small_drum():
    sc = S.drum(n=300, radius=25e-3, length=30e-3, n_boxes=32)
    target = np.array([0.0, -25e-3, 15e-3])
    sc.particles["velocity"] = sc.particles["velocity"] + (target - sc.particles["position"]) / 0.006
    return sc


@pytest.mark.parametrize("case", ["spheres", "drum"])
def test_persistent_steps_give_identical_runs(gpu_lib, case):
    """The middle steps in one cooperative launch (grid barriers between the
    phases) against the launched pipeline replayed from graphs: the same device
    bodies in the same order, hence identical bits (spheres with walls; convex
    bodies in the rotating drum, whose obstacles move inside the launch)."""
    sc = evolved_box() if case == "spheres" else small_drum()
    prec = FP64 if case == "spheres" else MIXED
    runs = []
    for persistent in (0, 1):
        s = make(gpu_lib, sc, prec)
        s.set_tuning(gather_every=5, persistent=persistent)
        s.initialize_leapfrog(0.0, sc.dt)
        t = s.step(37, 0.0, sc.dt)
        s.step(26, t, sc.dt)
        d = s.download()
        d["obstacles"] = s.obstacles(0, len(sc.obstacles[0]))
        runs.append(d)
        assert s.stats()["status"] == 0
        s.close()
    for k in ["position", "velocity", "omega", "force", "obstacles"]:
        assert np.array_equal(runs[0][k], runs[1][k]), k


def test_persistent_barrier_wait_runs_out_and_the_context_recovers(gpu_lib):
    """The persistent launch's grid barrier waits a bounded number of polls.
    With the test hook one block leaves before the first barrier and the wait
    bound is 1,000 polls: the other blocks' waits run out, GRAINS_GPU_TIMEOUT
    comes back through the status word (no fault, no hang), and the same
    context then runs the steps again to the bits of a fresh context."""
    from pacific_b200.abi import TIMEOUT, GrainsError
    sc = evolved_box()
    s = make(gpu_lib, sc, FP64)
    s.set_tuning(persistent=1)
    s.set_barrier_test(polls=1000, skip_block=0)
    s.initialize_leapfrog(0.0, sc.dt)
    with pytest.raises(GrainsError) as err:
        s.step(20, 0.0, sc.dt)
        s.synchronize()
    assert err.value.code & TIMEOUT
    # recovery: default bound, status cleared, state uploaded again
    s.set_barrier_test()
    s.reset_stats()
    s.update(sc.particles)
    s.upload_contact_memory({k: np.zeros((0, 3)) if k in ("kdelta", "prev_normal", "spring_torque")
                             else np.zeros(0, np.int32) for k in ("owner", "other", "kdelta", "prev_normal",
                                                                  "spring_torque")})
    s.initialize_leapfrog(0.0, sc.dt)
    s.step(20, 0.0, sc.dt)
    s.synchronize()
    assert s.stats()["status"] == 0
    fresh = make(gpu_lib, sc, FP64)
    fresh.set_tuning(persistent=1)
    fresh.initialize_leapfrog(0.0, sc.dt)
    fresh.step(20, 0.0, sc.dt)
    a, b = s.download(), fresh.download()
    for k in ["position", "velocity", "omega"]:
        assert np.array_equal(a[k], b[k]), k
