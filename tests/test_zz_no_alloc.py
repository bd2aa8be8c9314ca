"""The allocation-free contact detection (grains_gpu_sphere_contacts_noalloc)
gives the same contact pairs as the context-based path.

Some callers cannot call cudaMalloc -- code inside a stream capture that must
not allocate, real-time loops that cannot take cudaMalloc's implicit device
synchronisation, hosts that own all device memory through their own pool.
This entry point keeps its scratch in a fixed device array of the library and
only reads the caller's inputs and writes the caller's outputs.  The test
calls it twice in a row through the C ABI (different states, so the second
call must not see the first call's scratch) and compares each result with
the contact pairs of grains_gpu_compute_forces on the same state: the pair
sets are decided in double precision by both paths and must be identical.
This file is collected last so that a failure here stops a -x run only after
every other test has run."""
import ctypes as C

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64

from helpers import make, pair_set

pytestmark = pytest.mark.gpu


def noalloc_pairs(lib, sc, position, torch, cell_size=None, expect_status=0):
    fn = lib.dll.grains_gpu_sphere_contacts_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                   C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    n = sc.n
    dev = torch.device("cuda:0")
    pos = torch.tensor(np.ascontiguousarray(position).reshape(-1), dtype=torch.float64, device=dev)
    rad = torch.tensor(np.ascontiguousarray(sc.particles["radius"]), dtype=torch.float64, device=dev)
    cap = 16 * n
    pairs = torch.full((2 * cap,), -1, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    status = torch.full((1,), 12345, dtype=torch.int32, device=dev)
    d = sc.domains[0]
    origin = (C.c_double * 3)(*[float(x) for x in d["origin"]])
    size = (C.c_double * 3)(*[float(x) for x in d["size"]])
    stream = torch.cuda.current_stream(dev)
    cs = float(d["cell_size"]) if cell_size is None else cell_size
    rc = fn(n, pos.data_ptr(), rad.data_ptr(), origin, size, cs, pairs.data_ptr(), cap,
            count.data_ptr(), status.data_ptr(), stream.cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    k = int(count.item())
    assert 0 < k <= cap
    assert int(status.item()) == expect_status
    return pairs[: 2 * k].cpu().numpy().reshape(-1, 2)


def test_noalloc_contacts_match_context_path(gpu_lib):
    torch = pytest.importorskip("torch")
    sc = S.dense_cluster(343, seed=3, velocity_sigma=0.2)
    sim = make(gpu_lib, sc, FP64)
    # call 1: the initial state
    sim.compute_forces(0.0, sc.dt)
    expected = pair_set(sim.contact_pairs())
    got = noalloc_pairs(gpu_lib, sc, sc.particles["position"], torch)
    assert len(expected) > 500
    assert pair_set(got) == expected and len(got) == len(expected)
    # call 2: a state 40 steps later (particles moved to other cells)
    sim.initialize_leapfrog(0.0, sc.dt)
    sim.step(40, 0.0, sc.dt)
    sim.compute_forces(40 * sc.dt, sc.dt)
    state = sim.download()
    expected2 = pair_set(sim.contact_pairs())
    got2 = noalloc_pairs(gpu_lib, sc, state["position"], torch)
    assert expected2 != expected
    assert pair_set(got2) == expected2 and len(got2) == len(expected2)


def test_noalloc_rejects_oversized_input(gpu_lib):
    fn = gpu_lib.dll.grains_gpu_sphere_contacts_noalloc
    fn.restype = C.c_int
    origin = (C.c_double * 3)(0.0, 0.0, 0.0)
    size = (C.c_double * 3)(1.0, 1.0, 1.0)
    dummy = C.c_void_p(8)  # never dereferenced: the size check comes first
    rc = fn(C.c_int32(70000), dummy, dummy, origin, size, C.c_double(0.1), dummy, C.c_int64(1), dummy, dummy, None)
    assert rc != 0
    rc = fn(C.c_int32(10), dummy, dummy, origin, size, C.c_double(1e-3), dummy, C.c_int64(1), dummy, dummy, None)
    assert rc != 0  # 1e9 cells > 262,144
    # a cell count per axis above INT_MAX must be rejected before any
    # conversion to int (it would wrap to a negative product of counts)
    long_size = (C.c_double * 3)(1e4, 1e-6, 1e-6)
    rc = fn(C.c_int32(10), dummy, dummy, origin, long_size, C.c_double(1e-6), dummy, C.c_int64(1), dummy, dummy,
            None)
    assert rc != 0
    for bad in [float("nan"), float("inf"), -1.0]:
        rc = fn(C.c_int32(10), dummy, dummy, origin, size, C.c_double(bad), dummy, C.c_int64(1), dummy, dummy, None)
        assert rc != 0


def test_noalloc_flags_cells_smaller_than_a_diameter(gpu_lib):
    """A cell edge below the largest diameter can hide contacts two cells
    apart: the call still runs and reports GRAINS_GPU_CELL_TOO_SMALL."""
    torch = pytest.importorskip("torch")
    from pacific_b200.abi import CELL_TOO_SMALL
    sc = S.dense_cluster(343, seed=3, velocity_sigma=0.2)
    r_max = float(np.max(sc.particles["radius"]))
    # an edge just below the largest diameter: contacts along a diagonal of
    # neighbouring cells are still found, so some pairs come back
    got = noalloc_pairs(gpu_lib, sc, sc.particles["position"], torch, cell_size=1.9 * r_max,
                        expect_status=CELL_TOO_SMALL)
    sim = make(gpu_lib, sc, FP64)
    sim.compute_forces(0.0, sc.dt)
    assert pair_set(got) <= pair_set(sim.contact_pairs())
