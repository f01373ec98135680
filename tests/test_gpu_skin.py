"""The active pair list (skin) changes no result: a pair left out of it is farther
than 2R + skin at the last refresh and cannot have moved into contact since, so its
force is exactly zero, and every cell's row sum runs over the same shares in the
same order.  Runs with and without the skin must end bit for bit equal, in a static
state and in a growing one where the list is refreshed along the way."""
import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

pytestmark = pytest.mark.gpu
JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)


def run(cells, iters, skin, **kw):
    s = abm_b200.Simulation(cap_cells=len(cells) + 16, jkr_table=JKR, pair_skin=skin, **kw)
    s.upload_cells(cells)
    s.get_cell_neighbors()
    s.iterate(iters)
    out = s.download_cells(), s.clock(), s.stats()
    s.close()
    return out


@pytest.mark.parametrize("growth", [0.0, 1.5])
def test_skin_changes_no_result(growth):
    n = 3000
    cells, _ = workloads.biofilm_3d(n=n, seed=17, disk_radius=300.0 * np.sqrt(n / 1e5), p_contact=0.9)
    cells[:, 16] = growth
    cells[:, 13] = np.minimum(cells[:, 13], 4.0)
    cells[:, 14] = cells[:, 13] / 2
    kw = dict(max_stepsize=1e-3 if growth else 1e-5, iter_update_neighbors=100)
    a, ca, sa = run(cells, 150, 0.3, **kw)
    b, cb, sb = run(cells, 150, -1.0, **kw)
    c, cc, sc = run(cells, 150, 0.05, **kw)
    assert np.array_equal(a, b) and np.array_equal(a, c)
    assert ca == cb == cc
    assert sa["attempts"] == sb["attempts"] == sc["attempts"]


def test_skin_changes_no_result_2d_with_adhesion():
    cells = workloads.biofilm_2d(2000, seed=18, lmax=4.0)
    cells[:, 12] = 1.5
    kw = dict(abm_b200.DEFAULTS_2D, max_stepsize=1e-3, iter_update_neighbors=100, adhesion_mode=1,
              adhesion_strength=20.0, adhesion_mindist=1.2, Ldiv=4.4, neighbor_threshold=3.2)
    outs = []
    for skin in (0.3, -1.0):
        s = abm_b200.Simulation(cap_cells=2100, pair_skin=skin, **kw)
        s.upload_cells(cells)
        s.get_cell_neighbors()
        s.iterate(120)
        outs.append(s.download_cells())
        s.close()
    assert np.array_equal(outs[0], outs[1])
