"""pacific_b200 -- the Grains3D DEM time step (tortotubus/PacIFiC) on NVIDIA B200.

The compute path is the sm_100a shared library built from csrc/ into
lib/libgrains_gpu.so (python -m pacific_b200.build); Python only binds its C
ABI.  There is no CPU fallback: `load_library()` raises when the library is
missing or no CUDA device is usable.
"""
import os

from .abi import (BOX, CYLINDER, FP64, HERTZ, HERTZ_MEMORY, HOOKE, HOOKE_MEMORY, MIXED, POLYHEDRON, SPHERE, ContactError,  # noqa: F401
                  GrainsError, GrainsLib, MotionError, Simulation, SimulationError)

__version__ = "0.1.0"

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libgrains_gpu.so")
_LIB = None


def load_library(path=None):
    """Loads the CUDA implementation of the grains_gpu C ABI."""
    global _LIB
    if path is None and _LIB is not None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("pacific_b200: CUDA library not built (%s); run python -m pacific_b200.build" % p)
    lib = GrainsLib(p, "grains_gpu_")
    if path is None:
        _LIB = lib
    return lib
