"""Long-run statistics of the config-0 settling case against the reference.

1,000 spheres (r = 1 mm) dropped in a closed 20x20x60 mm box, HookeMemory,
dt = 1e-5 s, run for 30,000 steps: the configuration's 10,000 steps, in which
the spheres fall and pile up, and 20,000 more in which the bed comes to rest.
The reference's own run (tests/golden/settling_1k_stats.npz, made by
tests/golden/make_settling_stats.py with the reference built from its sources)
records every 500 steps the kinetic energy, the mean height and the mean
coordination number (Particle.cpp:1703-1707), and at the end the packing
fraction of the bed and the run statistics of AppCollision::addToContactsFeatures
(AppCollision.cpp:160-187): the largest and the mean overlap of every contact.

Granular flow is chaotic, so the runs are compared statistically, over windows
of the history.  The bars are about twice the spread between two independent
FP64 implementations of the reference's algorithm (the reference and the CPU
oracle, whose sums run in another order): kinetic energy within 2 % while the
spheres fall (steps 0-5,000) and 10 % during the pile-up (5,000-10,000), within
a factor 2 once at rest (there it is residual rattling, 1e-7 J); mean
coordination within 10 % during the pile-up and 25 % at rest (contacts at
rest carry overlaps of 1e-8 m and flicker); mean height at rest within 2 %;
packing fraction within 4 %; overlap maximum within 30 % and overlap mean within
10 %.  Both precisions are held to the same bars."""
import os
import sys

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def window(h, a, b, col):
    m = (h[:, 0] > a) & (h[:, 0] <= b)
    return float(h[m, col].mean())


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_settling_statistics_match_the_reference(gpu_lib, precision):
    import make_settling_stats as M
    ref = np.load(os.path.join(HERE, "golden", "settling_1k_stats.npz"))
    hr = ref["history"]
    hg, phi, omax, omean = M.run(gpu_lib, S.settling_1k(), precision)
    assert np.array_equal(hg[:, 0], hr[:, 0])
    KE, Z, COORD = 1, 2, 3

    def rel(a, b):
        return abs(a - b) / abs(b)
    assert rel(window(hg, 0, 5000, KE), window(hr, 0, 5000, KE)) < 0.02
    assert rel(window(hg, 5000, 10000, KE), window(hr, 5000, 10000, KE)) < 0.10
    ke_rest, ke_rest_ref = window(hg, 20000, 30000, KE), window(hr, 20000, 30000, KE)
    assert 0.5 < ke_rest / ke_rest_ref < 2.0
    assert rel(window(hg, 5000, 10000, COORD), window(hr, 5000, 10000, COORD)) < 0.10
    assert rel(window(hg, 20000, 30000, COORD), window(hr, 20000, 30000, COORD)) < 0.25
    assert rel(window(hg, 20000, 30000, Z), window(hr, 20000, 30000, Z)) < 0.02
    assert rel(phi, float(ref["packing_fraction"])) < 0.04
    assert rel(omax, float(ref["overlap_max"])) < 0.30
    assert rel(omean, float(ref["overlap_mean"])) < 0.10
