"""The C++ adaptor of include/grains_gpu.hpp (reference-style LinkedCellGPU,
Convex, ContactForceModel and exception classes) driving the step from a
compiled C++ program: spheres settle in a closed box, and a particle thrown
faster than its crust allows raises the reference's MotionError."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_host_example():
    exe = os.path.join(ROOT, "pacific_b200", "lib", "grains_host_example")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout.strip().splitlines()[-1])
    assert abs(d["time"] - 0.02) < 1e-12
    assert 0.0009 < d["zmin"] < 0.0012          # the bottom layer rests on the floor
    assert d["zmax"] < 0.0115                   # the column has fallen
    assert d["contacts"] > 0
    assert d["motion_error"] is True
