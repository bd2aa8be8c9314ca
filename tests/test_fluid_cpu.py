"""The DEM side of the fluid coupling in the oracle against the reference
itself (oracle/_ref): immersed particles with the buoyant weight
m (1 - rho_f / rho_p) g, the coupling factor 1 - rho_f / rho_p on the
translational and angular accelerations (Particle.cpp:414-419,
ParticleKinematics.cpp:483-488, SecondOrderLeapFrog.cpp:44-95,
ParticleKinematics3D.cpp:56-75) and the fluid's force and torque on every
particle (the reference's own AppPRSHydroFT registered after the collision
App, Fluid/src/AppPRSHydroFT.cpp:29-73).  Convex bodies: positions and
velocities bit for bit after 100 steps.  Spheres of a shaken box: the oracle
and the reference already differ by one unit in the last place of a velocity
without any fluid after 30 steps (1e-16 m/s, 4e-19 m after 100 steps), which
the fluid's torques amplify to 2e-12 m/s: positions within 1e-15 m, velocities
within 1e-11 m/s after 100 steps.  Skipped where the reference library is not
built."""
import os

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import GrainsLib

from helpers import make

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(REF_SO):
        pytest.skip("the reference library is not built (needs the reference sources)")
    return GrainsLib(REF_SO, "grains_ref_")


def immersed(sc, seed):
    """Particle densities (the scenarios' 2500 kg/m3) and seeded hydrodynamic
    forces and torques of the order of the weights."""
    rng = np.random.default_rng(seed)
    n = sc.n
    w = float(np.mean(sc.particles["mass"])) * 9.81
    return (np.full(n, 2500.0), rng.normal(0.0, 0.3 * w, size=(n, 3)),
            rng.normal(0.0, 0.3 * w * 1e-3, size=(n, 3)))


def run(lib, sc, fluid, corrected, rho, force, torque, steps=100):
    s = make(lib, sc)
    s.set_fluid(fluid, corrected, rho)
    s.set_hydro_forces(force, torque)
    s.initialize_leapfrog(0.0, sc.dt)
    s.step(steps, 0.0, sc.dt)
    d = s.download()
    s.close()
    return d


@pytest.mark.parametrize("corrected", [True, False], ids=["corrected", "uncorrected"])
@pytest.mark.parametrize("case", ["spheres", "convex"])
def test_immersed_particles_match_the_reference(oracle_lib, ref_lib, case, corrected):
    sc = S.small_box(125, seed=9, velocity_sigma=0.2) if case == "spheres" else S.convex_box(64, seed=4)
    rho, force, torque = immersed(sc, 1)
    a = run(ref_lib, sc, 1000.0, corrected, rho, force, torque)
    b = run(oracle_lib, sc, 1000.0, corrected, rho, force, torque)
    if case == "convex":
        for k in ["position", "velocity", "omega"]:
            assert np.array_equal(a[k], b[k]), k
    else:
        assert np.max(np.abs(a["position"] - b["position"])) < 1e-15
        assert np.max(np.abs(a["velocity"] - b["velocity"])) < 1e-11
    # the fluid changed the run
    c = run(oracle_lib, sc, 0.0, corrected, None, None, None)
    assert np.max(np.abs(c["velocity"] - b["velocity"])) > 1e-3
