"""The reload-file and RawData writers of the CUDA library: byte-for-byte
against files the reference itself wrote from the same state
(tests/golden/io_*.npz), the device formatter against C's printf, and
write -> read round trips of a 50,653-particle packed state after steps."""
import glob
import os

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED, format_doubles_on_device, read_reload_particles

from helpers import RAW_FILES, load_fixture_state, make, read_fixture_reload
from test_io_cpu import formatter_values, printf_form

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
IO_CASES = sorted(glob.glob(os.path.join(HERE, "golden", "io_*.npz")))
IDS = [os.path.basename(c)[:-4] for c in IO_CASES]


def test_device_formatter_matches_printf(gpu_lib):
    if "format_doubles" not in gpu_lib.fn:
        pytest.skip("the oracle has no device formatter")
    rng = np.random.default_rng(7)
    base = formatter_values(200000, 3)
    base += list(np.frombuffer(rng.integers(0x3c00000000000000, 0x4400000000000000, 100000, dtype=np.int64)
                               .astype(np.uint64).tobytes(), dtype=np.float64))
    for p in (16, 6):
        # the device formatter's range: 10^(p-87) <= |x| < 10^(p+28) (the writers format the rest on the host)
        vals = [x for x in base if np.isfinite(x) and (x == 0 or 10.0 ** (p - 86) < abs(x) < 10.0 ** (p + 27))]
        lines = format_doubles_on_device(gpu_lib, vals, p).split("\n")[:-1]
        assert len(lines) == len(vals)
        for x, s in zip(vals, lines):
            assert s == printf_form(float(x), p), (p, repr(x), s)


def test_values_outside_the_device_range_fall_back_to_the_host(oracle_lib, gpu_lib, tmp_path):
    """Huge, tiny, infinite and signed-zero values: the device defers the whole
    file to the host formatter, and the bytes equal the oracle's."""
    sc = S.dense_cluster(27, seed=2)
    p = dict(sc.particles)
    p["velocity"] = np.array(p["velocity"])
    p["omega"] = np.array(p["omega"], dtype=float)
    p["velocity"][3] = [3.7e45, -1e-200, -0.0]
    p["omega"][5] = [np.inf, -np.inf, 1e300]
    p["force"] = np.zeros((sc.n, 3))
    p["torque"] = np.zeros((sc.n, 3))
    p["force"][7] = [-0.0, 5e-324, 1.0]
    sc.particles = p
    outs = []
    for lib in (oracle_lib, gpu_lib):
        sim = make(lib, sc, FP64)
        path = os.path.join(str(tmp_path), "out_%d.txt" % len(outs))
        sim.write_reload_particles(path)
        root = os.path.join(str(tmp_path), "raw_%d" % len(outs))
        sim.write_rawdata(root, 0.0, truncate=True)
        outs.append([open(path, "rb").read()] + [open(root + f, "rb").read() for f in RAW_FILES])
        sim.close()
    assert outs[0] == outs[1]
    assert ("%.16e" % 3.7e45).encode() in outs[1][0] and b" inf " in outs[1][0] and b" -0 " in outs[1][0]


@pytest.mark.parametrize("path", IO_CASES, ids=IDS)
def test_reload_writer_matches_reference(reader_lib, gpu_lib, path, tmp_path):
    z = np.load(path)
    r = read_fixture_reload(reader_lib, z, tmp_path)
    _, sim = load_fixture_state(gpu_lib, z, r, FP64)
    for binary, key in [(False, "reload_text"), (True, "reload_bin")]:
        out = os.path.join(str(tmp_path), "gpu_" + key)
        nb = sim.write_reload_particles(out, binary=binary)
        data = open(out, "rb").read()
        assert nb == len(data)
        assert data == bytes(z[key]), key
    sim.close()


@pytest.mark.parametrize("path", IO_CASES, ids=IDS)
def test_rawdata_writer_matches_reference(reader_lib, gpu_lib, path, tmp_path):
    z = np.load(path)
    r = read_fixture_reload(reader_lib, z, tmp_path)
    sc, sim = load_fixture_state(gpu_lib, z, r, FP64)
    sim.compute_forces(float(z["time"]), sc.dt)  # coordination numbers of the state
    for binary, key in [(False, "raw_text"), (True, "raw_bin")]:
        root = os.path.join(str(tmp_path), "gpu_" + key)
        sim.write_rawdata(root, float(z["time"]), n_total=int(z["n_total"]), binary=binary, truncate=True)
        sim.write_rawdata(root, float(z["later"]), n_total=int(z["n_total"]), binary=binary, truncate=False)
        for f in RAW_FILES:
            assert open(root + f, "rb").read() == bytes(z[key + f]), key + f
    sim.close()


def memory_both_sides(mem):
    """(owner, other) -> 9 values over both sides of every particle pair and
    the particles' sides of their obstacle contacts (the particle file holds
    particles' maps only)."""
    out = {}
    for k in range(len(mem["owner"])):
        v = np.concatenate([mem["kdelta"][k], mem["prev_normal"][k], mem["spring_torque"][k]])
        a, b = int(mem["owner"][k]), int(mem["other"][k])
        if a < 0:
            continue
        out[(a, b)] = v
        if b >= 0:
            out.setdefault((b, a), -v)
    return out


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_round_trip_after_steps_50k(reader_lib, gpu_lib, precision, tmp_path):
    """50,653 spheres of a packed lattice (every neighbour and the walls in
    contact, about 120 MB of text: several 32 MB staging chunks) after 50
    steps on the device: the text and hybrid particle files read back to
    exactly the downloaded state and memory, and RawData rows to the state at
    6 digits."""
    sc = S.dense_cluster(50_653, seed=5, velocity_sigma=0.05)
    sim = make(gpu_lib, sc, precision, history_capacity=16)
    sim.initialize_leapfrog(0.0, sc.dt)
    t = sim.step(50, 0.0, sc.dt)
    st = sim.download()
    mem = memory_both_sides(sim.contact_memory(cap=1_000_000))
    assert len(mem) > 100_000
    for binary in (False, True):
        path = os.path.join(str(tmp_path), "save" + (".bin" if binary else ".txt"))
        sim.write_reload_particles(path, binary=binary)
        r = read_reload_particles(reader_lib, path, binary)
        assert np.array_equal(r["id"], st["id"])
        for k in ["position", "quaternion", "velocity", "omega", "force", "torque"]:
            assert np.array_equal(r[k], st[k]), k
        assert np.array_equal(r["basis"], st["basis"])
        assert np.all(r["transform_type"] == 3) and np.all(r["active"] == 1) and np.all(r["tag"] == 0)
        got = {(int(a), int(b)): np.concatenate([r["memory"]["kdelta"][k], r["memory"]["prev_normal"][k],
                                                 r["memory"]["spring_torque"][k]])
               for k, (a, b) in enumerate(zip(r["memory"]["owner"], r["memory"]["other"]))}
        assert set(got) == set(mem)
        for key, v in mem.items():
            assert np.array_equal(got[key], v), key
    root = os.path.join(str(tmp_path), "raw")
    sim.write_rawdata(root, t, truncate=True)
    row = open(root + "_position_x.dat").read().split()
    assert row[0] == printf_form(t, 6)
    order = np.argsort(st["id"])
    ids = st["id"][order]
    x = st["position"][order, 0]
    # ids 0..n-1 here: column i is id i + 1, so the last particle's column is absent (inactive)
    for i in range(0, sc.n - 1, 997):
        assert row[1 + i] == printf_form(float(x[ids == i + 1][0]), 6)
    assert row[sc.n] == printf_form(-1e10, 6)
    sim.close()
