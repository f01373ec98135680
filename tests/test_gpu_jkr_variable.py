"""The variable-gamma JKR table on the device (IsotropicJKRDataVariableGamma,
mechanics.hpp:159-199; forcesIsotropicJKRLagrange, adhesion.hpp:412-526): pair forces,
velocities and RK steps of a colony whose cells carry different gamma, against the
oracle's restatement, through the C ABI.  Bars: 1e-10 normwise (FP64), 1e-4 (mixed)."""
import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

pytestmark = pytest.mark.gpu

MAX_GAMMA = 120.0


def colony(n=3000, seed=51):
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=300.0 * np.sqrt(n / 1e5), p_contact=0.9)
    rng = np.random.default_rng(seed)
    # a mix of gamma values: zero (no adhesion), the top of the mesh, between mesh points
    g = rng.uniform(0.0, MAX_GAMMA, size=n)
    g[rng.random(n) < 0.15] = 0.0
    g[rng.random(n) < 0.15] = MAX_GAMMA
    cells[:, 21] = g
    return cells


def colwise_relerr(a, b):
    scale = np.abs(b).max(axis=0)
    diff = np.abs(a - b).max(axis=0)
    return float(np.max(np.where(scale > 0, diff / np.where(scale > 0, scale, 1), diff)))


@pytest.mark.parametrize("precision", [abm_b200.PRECISION_FP64, abm_b200.PRECISION_MIXED])
def test_variable_gamma_forces_and_step_match_oracle(precision):
    cells = colony()
    d, g, r = abm_b200.jkr_radius_table_variable(0.8, 0.5, 3900.0, MAX_GAMMA, 100, 60)
    sim = abm_b200.Simulation(cap_cells=len(cells), precision=precision,
                              jkr_table=orc.jkr_table(0.8, 0.5, 3900.0, 1.0))
    sim.set_jkr_table_variable(d, g, r)
    sim.upload_cells(cells)
    o = orc.Oracle(sim.pdict)
    o.set_jkr_table_variable(d, g, r)
    o.set_cells(cells)
    assert sim.get_cell_neighbors() == o.build_neighbors()
    tol = 1e-10 if precision == abm_b200.PRECISION_FP64 else 1e-4
    fo = o.cell_cell_forces()
    assert colwise_relerr(sim.cell_cell_forces(), fo) <= tol
    # the table matters: the forces differ from those of one fixed gamma
    fixed = abm_b200.Simulation(cap_cells=len(cells), jkr_table=orc.jkr_table(0.8, 0.5, 3900.0, MAX_GAMMA))
    fixed.upload_cells(cells)
    fixed.get_cell_neighbors()
    assert colwise_relerr(fixed.cell_cell_forces(), fo) > 1e-3
    fixed.close()
    assert colwise_relerr(sim.get_velocities(), o.get_velocities()) <= tol
    cg, _, Eg = sim.step_runge_kutta_adaptive(1e-6)
    co, _, Eo = o.rk_attempt(1e-6)
    assert colwise_relerr(cg, co) <= tol
    sim.close()


def test_fixed_table_after_variable_restores_the_fixed_forces():
    cells = colony(1500, 52)
    jkr = orc.jkr_table(0.8, 0.5, 3900.0, 100.0)
    ref = abm_b200.Simulation(cap_cells=len(cells), jkr_table=jkr)
    ref.upload_cells(cells)
    ref.get_cell_neighbors()
    expect = ref.cell_cell_forces()
    sim = abm_b200.Simulation(cap_cells=len(cells), jkr_table=jkr)
    sim.set_jkr_table_variable(*abm_b200.jkr_radius_table_variable(0.8, 0.5, 3900.0, MAX_GAMMA, 100, 40))
    sim.set_jkr_table(*jkr)
    sim.upload_cells(cells)
    sim.get_cell_neighbors()
    assert np.array_equal(sim.cell_cell_forces(), expect)
    ref.close()
    sim.close()
