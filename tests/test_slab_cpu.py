"""The slab decomposition (pacific_b200/slab.py) on two processes with the gloo
backend, each rank stepping its slab and ghosts with the CPU oracle, against
the same scenario stepped as one domain: every particle's final state from its
owner, after runs in which particles change owner at the rebuilds.

The ghost refresh writes only the ghosts (grains_gpu_update_particle_rows), so
a run without rebuilds follows the single domain bit for bit until the force
sums, whose order depends on which particles a rank holds, first round
differently.  A rebuild re-uploads every particle, and the upload derives the
body-frame angular velocity from the world one, one more rounding.  The dense,
shaken packings amplify such differences about a thousandfold every 50 steps
(spheres: 1e-19 m after 10 steps, 6e-15 m after 50, 3e-11 m after 100; the
convex cluster: exact for 10 steps, 7e-11 m after 20, 5e-10 m after 40), so
the bars are 1e-9 m after 100 steps for spheres and 1e-8 m after 40 steps for
the convex cluster, with a rebuild every 10 steps (particles change owner at
the rebuilds) or on drift.  The convex runs use the order-independent
polyhedron support rule of the CUDA path (oracle mode 2) on both sides."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from pacific_b200 import scenarios as S

from helpers import make

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libgrains_oracle.so")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def scenario(name, oracle_lib=None):
    """The scenario, the steps, the rebuild period, the drift bound and the
    initial contact memory."""
    if name == "spheres":
        return S.small_box(343, seed=11, velocity_sigma=0.5), 100, 10, None, None
    if name == "drift":
        # rebuilds forced by the drift bound alone (0.01 mm; the fastest
        # spheres move 0.02 mm in 10 steps)
        return S.small_box(343, seed=12, velocity_sigma=0.5), 100, 1000, 1e-5, None
    # cubes, cylinders and octahedra of a converging cluster, advanced by the
    # oracle into contact first (with its contact memory)
    from pacific_b200.abi import GrainsLib
    lib = oracle_lib or GrainsLib(ORACLE_SO, "grains_oracle_")
    sc = S.convex_box(125, seed=3, converge_time=2e-3)
    o = make(lib, sc)
    o.initialize_leapfrog(0.0, sc.dt)
    o.step(500, 0.0, sc.dt)
    st, mem = o.download(), o.contact_memory()
    o.close()
    p = dict(sc.particles)
    for k in ["position", "quaternion", "basis", "velocity", "omega"]:
        p[k] = st[k]
    sc.particles = p
    return sc, 40, 10, None, mem


def rank_main(rank, world, port, name, out_dir):
    import torch.distributed as dist
    from pacific_b200.abi import FP64, GrainsLib
    from pacific_b200.slab import SlabRun
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lib = GrainsLib(ORACLE_SO, "grains_oracle_")
        sc, steps, every, drift, mem = scenario(name, lib)
        run = SlabRun(lib, sc, FP64, rebuild_every=every, drift=drift, memory=mem)
        run.sim.set_polyhedron_support(2)
        if mem is None:
            run.initialize_leapfrog(0.0, sc.dt)
        owned0 = run.owned[rank].copy()
        run.step(steps, 0.0, sc.dt)
        g = run.gather()
        moved = len(np.setxor1d(owned0, run.owned[rank]))
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), position=g["position"], velocity=g["velocity"],
                 coordination=g["coordination"], rebuilds=run.rebuilds, changed=moved,
                 ghosts=len(run.ghosts[rank]), owned=len(run.owned[rank]))
        run.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["spheres", "drift", "convex"])
def test_slab_run_matches_one_domain(oracle_lib, name):
    sc, steps, _, _, mem = scenario(name, oracle_lib)
    one = make(oracle_lib, sc)
    one.set_polyhedron_support(2)
    if mem is None:
        one.initialize_leapfrog(0.0, sc.dt)
    else:
        one.upload_contact_memory(mem)
    one.step(steps, 0.0, sc.dt)
    ref = one.download()
    one.close()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(rank_main, args=(2, free_port(), name, d), nprocs=2, join=True, start_method="spawn")
        r0, r1 = (np.load(os.path.join(d, "r%d.npz" % k)) for k in range(2))
        # both ranks gathered the same full state
        assert np.array_equal(r0["position"], r1["position"])
        assert int(r0["owned"]) + int(r1["owned"]) == sc.n
        assert int(r0["ghosts"]) > 0 and int(r1["ghosts"]) > 0
        assert int(r0["rebuilds"]) >= 4
        assert int(r0["changed"]) + int(r1["changed"]) > 0  # particles changed owner
        assert np.max(np.abs(r0["position"] - ref["position"])) < (1e-9 if name != "convex" else 1e-8)
        assert np.max(np.abs(r0["velocity"] - ref["velocity"])) < (1e-5 if name != "convex" else 1e-4)
