"""Pins the forward-mode oracle of the adjoint (oracle/tangent_oracle.cpp):
its plain FP64 run follows the main oracle (itself pinned to the reference's
golden fixtures), and its dual-number derivatives equal central finite
differences of its own run.  512 spheres dropped with N(0, 0.2 m/s) velocities
for 100 steps: the first collisions, before the chaotic growth of
sensitivities (the tangent norm grows about tenfold per 10-20 steps once the
particles collide) makes finite differences leave their linear range."""
import numpy as np

from pacific_b200 import scenarios as S

from helpers import make, tangent_run

N, STEPS = 512, 100


def test_tangent_oracle_run_follows_the_oracle(oracle_lib):
    sc = S.adjoint_4k(n=N)
    fin, _ = tangent_run(sc, STEPS)
    o = make(oracle_lib, sc)
    o.initialize_leapfrog(0.0, sc.dt)
    o.step(STEPS, 0.0, sc.dt)
    d = o.download()
    # same double arithmetic except the angular velocity, integrated here in
    # the world frame instead of the body frame (equal for spheres up to rounding)
    assert np.max(np.abs(d["position"] - fin["position"])) < 1e-15
    assert np.max(np.abs(d["velocity"] - fin["velocity"])) < 1e-12
    assert np.max(np.abs(d["omega"] - fin["omega"])) < 1e-9
    assert np.max(np.abs(fin["velocity"] - sc.particles["velocity"])) > 0.01, "the spheres should collide"


def scaled(idx, delta):
    sc = S.adjoint_4k(n=N)
    sc.laws = [[(a, b, law, [p + delta if k == idx else p for k, p in enumerate(prm)]) for a, b, law, prm in sc.laws[0]]]
    return sc


def test_dual_derivatives_equal_finite_differences():
    sc = S.adjoint_4k(n=N)
    rng = np.random.default_rng(3)
    dv = np.zeros((6, N, 3))
    dv[4:] = rng.normal(size=(2, N, 3))
    dl = np.zeros((6, 16, 4))
    for t in range(4):
        dl[t, [0, 1, 4], t] = 1.0   # slots (0, 0), (0, 1), (1, 0): particle pairs and walls
    fin, tan = tangent_run(sc, STEPS, dv, dl)
    for t, idx in enumerate([0, 1, 3, 4]):  # kn, en, muc, kt in the HookeMemory parameter list
        h = 1e-6 * sc.laws[0][0][3][idx]
        fp, _ = tangent_run(scaled(idx, h), STEPS)
        fm, _ = tangent_run(scaled(idx, -h), STEPS)
        fd = (fp["velocity"] - fm["velocity"]) / (2 * h)
        assert np.max(np.abs(fd - tan["velocity"][t])) < 1e-5 * np.max(np.abs(fd)), t
    # velocity directions: h = 1e-8, where the difference quotient is clear of
    # the rare particle whose contact law changes branch (stick / slip) between
    # the two runs at 1e-7, and still above rounding
    for t in (4, 5):
        h = 1e-8
        scp, scm = S.adjoint_4k(n=N), S.adjoint_4k(n=N)
        scp.particles["velocity"] = scp.particles["velocity"] + h * dv[t]
        scm.particles["velocity"] = scm.particles["velocity"] - h * dv[t]
        fp, _ = tangent_run(scp, STEPS)
        fm, _ = tangent_run(scm, STEPS)
        fd = (fp["velocity"] - fm["velocity"]) / (2 * h)
        assert np.max(np.abs(fd - tan["velocity"][t])) < 1e-4 * np.max(np.abs(fd)), t
