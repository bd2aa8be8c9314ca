"""The pieces of the slab decomposition that run on the GPU, on the one GPU
of a test machine: grains_gpu_update_particle_rows against the whole-state
update, and a slab run of one rank (its rebuilds re-upload the particles and
their contact memory every 10 steps) against the plain run of the same steps
on the CUDA library.  The exchange between ranks is covered on the CPU
(tests/test_slab_cpu.py, two gloo ranks)."""
import os
import socket

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED

from helpers import make, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_update_rows_equals_whole_update(gpu_lib, precision):
    sc = S.small_box(343, seed=5, velocity_sigma=0.3)
    a, b = make(gpu_lib, sc, precision), make(gpu_lib, sc, precision)
    for s in (a, b):
        s.initialize_leapfrog(0.0, sc.dt)
        s.step(20, 0.0, sc.dt)
    st = a.download()
    rng = np.random.default_rng(0)
    rows = rng.choice(sc.n, size=60, replace=False)
    new = {k: st[k].copy() for k in ["position", "quaternion", "velocity", "omega"]}
    new["position"][rows] += rng.uniform(-2e-5, 2e-5, size=(60, 3))
    new["velocity"][rows] = rng.normal(0.0, 0.2, size=(60, 3))
    new["omega"][rows] = rng.normal(0.0, 20.0, size=(60, 3))
    a.update(new)
    b.update_rows(rows, {k: v[rows] for k, v in new.items()})
    da, db = a.download(), b.download()
    for k in ["position", "quaternion", "velocity", "omega"]:
        assert np.array_equal(da[k], db[k])
    for s in (a, b):
        s.compute_forces(20 * sc.dt, sc.dt)
    assert np.array_equal(a.download()["force"], b.download()["force"])
    with pytest.raises(Exception):
        b.update_rows(np.array([3, 3]), {k: v[[3, 3]] for k, v in new.items()})
    a.close()
    b.close()


def test_one_rank_slab_run_follows_the_plain_run(gpu_lib):
    import torch.distributed as dist
    from pacific_b200.slab import SlabRun
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        sc = S.small_box(343, seed=11, velocity_sigma=0.5)
        run = SlabRun(gpu_lib, sc, FP64, rebuild_every=10)
        run.initialize_leapfrog(0.0, sc.dt)
        run.step(60, 0.0, sc.dt)
        g = run.gather()
        run.close()
        assert run.rebuilds >= 6
        one = make(gpu_lib, sc, FP64)
        one.initialize_leapfrog(0.0, sc.dt)
        one.step(60, 0.0, sc.dt)
        ref = one.download()
        one.close()
        # the re-uploads at the rebuilds derive the body-frame angular velocity
        # again: rounding, amplified by the shaken box
        assert np.max(np.abs(g["position"] - ref["position"])) < 1e-10
        assert np.array_equal(g["coordination"], ref["coordination"])
        weight = float(np.min(sc.particles["mass"])) * 9.81
        assert rel_err(g["force"], ref["force"], weight) < 1e-4
    finally:
        dist.destroy_process_group()
