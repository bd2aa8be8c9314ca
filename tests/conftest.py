import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libgrains_oracle.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# GRAINS_SELFTEST_ORACLE=1 runs the GPU tests with the oracle standing in
# for the CUDA library (checks the test code itself on a CPU machine).
SELFTEST = os.environ.get("GRAINS_SELFTEST_ORACLE") == "1"


def pytest_collection_modifyitems(config, items):
    if _cuda_available() or SELFTEST:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s"], check=True)
    from pacific_b200.abi import GrainsLib
    return GrainsLib(ORACLE_SO, "grains_oracle_")


@pytest.fixture(scope="session")
def gpu_lib(oracle_lib):
    if SELFTEST:
        return oracle_lib
    import pacific_b200
    return pacific_b200.load_library()


@pytest.fixture(scope="session")
def reader_lib():
    """The CUDA library for its host-only entry points (reload reader, host
    formatter): loading it needs no device."""
    import pacific_b200
    return pacific_b200.load_library()
