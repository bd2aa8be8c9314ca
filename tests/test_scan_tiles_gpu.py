"""Cell lists of a grid that spans several tiles of the cell-count scan
(4,096 cells per tile): 8,000 spheres in a 44 x 44 x 66 mm box with 2 mm
cells (15,972 cells, four tiles).  The launched sort scans within tiles and
adds each tile's start in the scatter and the cell sort; the persistent launch
scans the whole grid in one pass of its own.  Both must give the same runs to
the bit, and the candidate pairs must be the oracle's."""
import math

import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64

from helpers import make

pytestmark = pytest.mark.gpu

SCAN_TILE = 4096


def multi_tile_box():
    sc = S.small_box(8000, seed=12, velocity_sigma=0.3)
    d = sc.domains[0]
    cells = 1
    for a in range(3):
        cells *= int(math.floor(d["size"][a] / d["cell_size"]))
    assert cells > 3 * SCAN_TILE
    return sc


def test_candidate_pairs_across_scan_tiles(oracle_lib, gpu_lib):
    sc = multi_tile_box()
    o, g = make(oracle_lib, sc), make(gpu_lib, sc, FP64)
    co = o.candidate_pairs(include_obstacles=True)
    cg = g.candidate_pairs(include_obstacles=True)
    assert len(co) > sc.n
    assert np.array_equal(co, cg)
    o.close()
    g.close()


def test_launched_and_persistent_sorts_agree_across_scan_tiles(gpu_lib):
    sc = multi_tile_box()
    runs = []
    for persistent in (0, 1):
        s = make(gpu_lib, sc, FP64)
        s.set_tuning(gather_every=5, persistent=persistent)
        s.initialize_leapfrog(0.0, sc.dt)
        t = s.step(37, 0.0, sc.dt)
        s.step(26, t, sc.dt)
        runs.append(s.download())
        assert s.stats()["status"] == 0
        s.close()
    for k in ["position", "velocity", "omega", "force", "coordination"]:
        assert np.array_equal(runs[0][k], runs[1][k]), k
    assert np.sum(runs[0]["coordination"]) > 0
