"""The reload-file and RawData formats on the CPU: the library's host
formatter against C's printf, its particle-file reader on files the reference
wrote, and the oracle's restatement of both writers against the reference's
bytes (tests/golden/io_*.npz, made by tests/golden/make_io_golden.py)."""
import glob
import os

import numpy as np
import pytest

from pacific_b200.abi import format_double

from helpers import RAW_FILES, load_fixture_state, read_fixture_reload

HERE = os.path.dirname(os.path.abspath(__file__))
IO_CASES = sorted(glob.glob(os.path.join(HERE, "golden", "io_*.npz")))
IDS = [os.path.basename(c)[:-4] for c in IO_CASES]


def printf_form(x, p):
    """GrainsExec::doubleToString(ios::scientific, p, x): %.{p}e, zeros as 0 / -0."""
    if x == 0.0:
        return "-0" if np.signbit(x) else "0"
    return "%.*e" % (p, x)


def formatter_values(n, seed):
    rng = np.random.default_rng(seed)
    v = list(rng.standard_normal(n) * 10.0 ** rng.integers(-75, 45, n))
    for s in range(0, 56):  # exact binary fractions: ties of the last digit
        v += [k / 2.0 ** s for k in (1, 3, 5, 7, 25, 125, 625, 3125)]
    for e in range(-70, 44):
        x = 10.0 ** e
        v += [x, np.nextafter(x, 0.0), np.nextafter(x, 1e308), 9.5 * 10.0 ** e, 0.99999999999999995 * 10.0 ** e]
    v += [0.0, -0.0, 1.0, -1.0, 1e-300, 1e300, 5e-324, 1.7976931348623157e308, float("inf"), -float("inf")]
    return [float(x) for x in v]


def test_host_formatter_matches_printf(reader_lib):
    for p in (16, 6):
        for x in formatter_values(20000, p):
            assert format_double(reader_lib, x, p) == printf_form(x, p), (p, repr(x))


@pytest.mark.parametrize("path", IO_CASES, ids=IDS)
def test_reader_text_and_binary_agree(reader_lib, path, tmp_path):
    """The reference's text and hybrid files of one state read back to the
    same values (the text carries 17 significant digits: exact)."""
    z = np.load(path)
    a = read_fixture_reload(reader_lib, z, tmp_path, binary=False)
    b = read_fixture_reload(reader_lib, z, tmp_path, binary=True)
    for k in ["geom_type", "id", "tag", "active", "transform_type", "position", "basis", "velocity", "quaternion",
              "omega", "force", "torque"]:
        assert np.array_equal(a[k], b[k]), k
    for k in a["memory"]:
        assert np.array_equal(a["memory"][k], b["memory"][k]), k
    assert len(a["id"]) == int(z["n_total"])
    assert len(a["memory"]["owner"]) > 0


@pytest.mark.parametrize("path", IO_CASES, ids=IDS)
def test_oracle_reload_writer_matches_reference(reader_lib, oracle_lib, path, tmp_path):
    z = np.load(path)
    r = read_fixture_reload(reader_lib, z, tmp_path)
    _, sim = load_fixture_state(oracle_lib, z, r)
    for binary, key in [(False, "reload_text"), (True, "reload_bin")]:
        out = os.path.join(str(tmp_path), "oracle_" + key)
        sim.write_reload_particles(out, binary=binary)
        assert open(out, "rb").read() == bytes(z[key]), key
    sim.close()


@pytest.mark.parametrize("path", IO_CASES, ids=IDS)
def test_oracle_rawdata_writer_matches_reference(reader_lib, oracle_lib, path, tmp_path):
    z = np.load(path)
    r = read_fixture_reload(reader_lib, z, tmp_path)
    sc, sim = load_fixture_state(oracle_lib, z, r)
    sim.compute_forces(float(z["time"]), sc.dt)  # coordination numbers of the state
    for binary, key in [(False, "raw_text"), (True, "raw_bin")]:
        root = os.path.join(str(tmp_path), "oracle_" + key)
        sim.write_rawdata(root, float(z["time"]), n_total=int(z["n_total"]), binary=binary, truncate=True)
        sim.write_rawdata(root, float(z["later"]), n_total=int(z["n_total"]), binary=binary, truncate=False)
        for f in RAW_FILES:
            assert open(root + f, "rb").read() == bytes(z[key + f]), key + f
    sim.close()
