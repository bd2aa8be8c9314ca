"""The CUDA path against the reference's own results (golden fixtures made by
the reference Grains3D built from its sources, tests/golden/make_golden.py).
Pair sets and coordination exact; plain FP64 forces within 1e-12 relative,
mixed precision within 1e-5 (force floor: the particle weight)."""
import glob
import os
import sys

import numpy as np
import pytest

from pacific_b200.abi import FP64, MIXED

from helpers import make, pair_set, rel_err

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
CASES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def test_gpu_matches_reference_fixture(gpu_lib, path, precision):
    import golden_io as G
    z = np.load(path)
    sc = G.scenario_from_npz(z)
    sim = make(gpu_lib, sc, precision)
    sim.upload_contact_memory(G.memory_from(z, "mem_in_"))
    t = float(z["time"])
    sim.compute_forces(t, sc.dt)
    d = sim.download()
    weight = float(np.min(sc.particles["mass"])) * 9.81
    assert np.array_equal(d["coordination"], z["coordination"])
    assert np.array_equal(sim.candidate_pairs(), z["candidate_pairs"])
    if bool(z["has_contact_pairs"]):
        assert pair_set(sim.contact_pairs()) == pair_set(z["contact_pairs"])
    tol = 1e-12 if precision == FP64 else 1e-5
    assert rel_err(d["force"], z["force"], weight) < tol
    assert rel_err(d["torque"], z["torque"], weight * 1e-3) < (1e-10 if precision == FP64 else 1e-5)
    # 20-40 further steps: FP64 stays at rounding level; in mixed precision the
    # FP32 rounding of forces is amplified by the chaotic dense-packing
    # dynamics (observed up to 3e-8 m after 20 steps of a dense cluster)
    steps = int(z["after_steps"])
    sim.step(steps, t, sc.dt)
    d = sim.download()
    assert np.max(np.abs(d["position"] - z["after_position"])) < (1e-13 if precision == FP64 else 2e-7)
