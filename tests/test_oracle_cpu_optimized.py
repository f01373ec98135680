"""The oracle's "optimized CPU" procedures, which time the context figure reported
beside the reference-faithful CPU run: a cell-list neighbor build and the pair forces
with OpenMP over the pairs.  The neighbor table must equal the reference's O(n^2)
getCellNeighbors (mechanics.hpp:520-593) entry for entry, and the forces and a loop
must agree with the faithful procedures to rounding (the parallel pair sums add in
another order)."""
import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)


def state(n, seed, radius=None, p_contact=0.9):
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=radius or 300.0 * np.sqrt(n / 1e5),
                                    p_contact=p_contact)
    return cells


def pair(cells, **kw):
    _, p = abm_b200.make_params(**kw)
    out = []
    for opt in (False, True):
        o = orc.Oracle(p, jkr=JKR, cpu_optimized=opt)
        o.set_cells(cells)
        out.append(o)
    return out


@pytest.mark.parametrize("n, seed, radius", [(3000, 1, None), (800, 2, 400.0), (2, 3, 1.0), (1, 4, 1.0), (0, 5, 1.0)])
def test_cell_list_table_equals_the_reference_procedure(n, seed, radius):
    cells = state(max(n, 1), seed, radius)[:n]
    a, b = pair(cells)
    ma, mb = a.build_neighbors(), b.build_neighbors()
    assert ma == mb
    assert np.array_equal(a.neighbors(), b.neighbors())
    if n == 3000:
        assert ma > 3 * n                     # the benchmark density: several pairs per cell


def test_parallel_pair_forces_agree_to_rounding():
    cells = state(4000, 7)
    a, b = pair(cells)
    a.build_neighbors(), b.build_neighbors()
    fa, fb = a.cell_cell_forces(), b.cell_cell_forces()
    scale = np.abs(fa).max(axis=0)
    assert np.all(scale > 0)
    assert (np.abs(fa - fb).max(axis=0) / scale).max() <= 1e-13


def test_optimized_loop_takes_the_faithful_decisions():
    cells = state(2000, 8)
    cells[:, 16] = 1.5
    a, b = pair(cells, max_stepsize=1e-4, growth_mean=1.5)
    for o in (a, b):
        o.loop_init()
        o.iterate(6)
    sa, sb = a.stats(), b.stats()
    for k in ("attempts", "rebuilds", "divisions", "rejected"):
        assert sa[k] == sb[k], k
    assert abs(sa["last_max_error"] - sb["last_max_error"]) <= 1e-9 * sa["last_max_error"]
    ca, cb = a.cells(), b.cells()
    scale = np.maximum(np.abs(ca).max(axis=0), 1e-300)
    assert (np.abs(ca - cb).max(axis=0) / scale).max() <= 1e-12
    (ta, da, ia), (tb, db, ib) = a.clock(), b.clock()
    assert ia == ib == 6 and abs(ta - tb) <= 1e-12 * ta and abs(da - db) <= 1e-12 * da
