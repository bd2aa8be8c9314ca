"""The reference's own time loop with the B200 collision App.

LinkedCellGPU (pacific_b200/reference_app/LinkedCellGPU.{hh,cpp}) is compiled
against the reference's headers into the reference library built from its own
sources (oracle/ref/Makefile -> oracle/_ref/libgrains_ref.so) and takes the
place of the reference's LinkedCell in a Grains simulation, the way
Grains::Construction registers its LinkedCell (Base/src/Grains.cpp:777-780).
The reference's Grains then runs its leapfrog (Grains::moveParticlesAndObstacles
-> LinkUpdate, Grains::computeParticlesForceAndTorque -> App::ComputeForces,
AllComponents::advanceParticlesVelocity; Grains.cpp:344-364, 459-527) on its
own list<Particle*>; only the collision App runs on the GPU.

Against the same simulation with the reference's stock LinkedCell: the
torsors of the leapfrog start within 1e-12 of the weight-floored force (the
GPU's contact forces differ from the reference's only by the order of
floating-point sums), positions within 1e-10 m after 40 steps of a dense
packing (where those rounding differences grow), and the same coordination
numbers."""
import ctypes as C
import os

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, GrainsLib

from helpers import make, rel_err

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")


@pytest.fixture(scope="module")
def ref_lib(gpu_lib):
    if not os.path.exists(REF_SO):
        pytest.skip("the reference library is not built (needs the reference sources)")
    return GrainsLib(REF_SO, "grains_ref_")


def run_reference(ref_lib, sc, device=None, steps=40):
    """The reference simulation of `sc` (its own leapfrog), with the GPU App
    over `device` when given; one reference simulation alive at a time (the
    reference keeps some of its tables in statics)."""
    s = make(ref_lib, sc)
    try:
        if device is not None:
            use = ref_lib.dll.grains_ref_use_gpu_app
            use.argtypes = [C.c_void_p, C.c_void_p]
            use.restype = C.c_int
            assert use(s.ctx, device.ctx) == 0
        s.initialize_leapfrog(0.0, sc.dt)
        first = s.download()
        s.step(steps, 0.0, sc.dt)
        return first, s.download()
    finally:
        s.close()


@pytest.mark.parametrize("case", ["dense_cluster", "small_box"])
def test_reference_time_loop_with_the_gpu_app(gpu_lib, ref_lib, case):
    sc = S.dense_cluster(216, seed=31, velocity_sigma=0.1) if case == "dense_cluster" else \
        S.small_box(343, seed=32, velocity_sigma=0.3, spacing=2.0)
    a0, a = run_reference(ref_lib, sc)
    device = make(gpu_lib, sc, FP64)
    b0, b = run_reference(ref_lib, sc, device)
    weight = float(np.min(sc.particles["mass"])) * 9.81
    # the leapfrog start (same state): the torsors at rounding level
    assert int(a0["coordination"].sum()) > 100
    assert rel_err(b0["force"], a0["force"], weight) < 1e-12
    assert rel_err(b0["torque"], a0["torque"], weight * 1e-3) < 1e-10
    # 40 steps of the reference's leapfrog: the rounding differences of the
    # force sums grow in a dense packing (6.5e-12 m measured on the dense case)
    assert np.max(np.abs(b["position"] - a["position"])) < 1e-10
    assert np.max(np.abs(b["velocity"] - a["velocity"])) < 1e-6
    # the device context saw the same contacts in its last evaluation
    assert np.array_equal(device.download()["coordination"], a["coordination"])
    device.close()
