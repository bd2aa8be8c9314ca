"""The library's narrowphase built for the host (tests/gjk_host_check.cpp):
the signed-volume GJK (Montanari, Petrinic and Barbieri 2017, in
pacific_b200/csrc/gjk.cuh) against closed-form distances and against
certified lower bounds on 40,000 seeded random pairs of boxes, cylinders and
octahedra; it must never reach the 1000-iteration cap."""
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def test_signed_volume_gjk_on_host():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "gjk_host_check")
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I/usr/local/cuda/include",
                        os.path.join(HERE, "gjk_host_check.cpp"), "-o", exe], check=True)
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "failures 0" in r.stdout
