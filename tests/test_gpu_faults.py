"""Failures injected from the host through the inputs, the counterparts of the
reference's DEBUG_CHECK_* guards (e.g. mechanics.hpp:759-777 for NaN cell
coordinates, simulation.hpp:1803-1821 for NaN velocities): each must come back as a
status code through the C ABI, and no kernel may write outside its buffers.

  * a NaN coordinate: ABM_ERR_NAN from the step (the error norm is NaN);
  * a division that would exceed cap_cells: ABM_ERR_CAPACITY, and no cell divides;
  * a colony no cell-list grid can hold (a coordinate at 1e295 or infinity):
    ABM_ERR_CAPACITY from the neighbor build, with an empty neighbor set;
  * more neighbors than cap_neighbors_per_cell: covered in test_gpu_parity.py.
"""
import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

pytestmark = pytest.mark.gpu

JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0)


def patch(n, seed):
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=300.0 * np.sqrt(n / 1e5), p_contact=0.9)
    return cells


@pytest.mark.parametrize("col", [1, 6])
def test_nan_coordinate_is_reported(col):
    cells = patch(500, 61)
    cells[7, col] = np.nan
    sim = abm_b200.Simulation(cap_cells=600, jkr_table=JKR)
    sim.upload_cells(cells)
    sim.get_cell_neighbors()
    with pytest.raises(RuntimeError, match="ABM_ERR_NAN"):
        sim.iterate(1)
    sim.close()
    sim = abm_b200.Simulation(cap_cells=600, jkr_table=JKR)
    sim.upload_cells(cells)
    sim.get_cell_neighbors()
    with pytest.raises(RuntimeError, match="ABM_ERR_NAN"):
        sim.step_runge_kutta_adaptive(1e-6)
    sim.close()


def test_division_past_capacity_is_reported():
    n = 300
    cells = patch(n, 62)
    cells[:, 13] = 5.7                      # every cell is past Ldiv = 5.6
    cells[:, 14] = 5.7 / 2
    sim = abm_b200.Simulation(cap_cells=n, jkr_table=JKR, growth_mean=1.5, growth_std=0.1,
                              daughter_length_std=0.05, daughter_angle_xy_bound=0.3, daughter_angle_z_bound=0.1)
    sim.upload_cells(cells)
    sim.set_parents(-np.ones(n, dtype=np.int32))
    sim.get_cell_neighbors()
    with pytest.raises(RuntimeError, match="ABM_ERR_CAPACITY.*cap_cells"):
        sim.iterate(1)
    assert sim.num_cells() == n
    assert np.isfinite(sim.download_cells()).all()
    sim.close()


@pytest.mark.parametrize("far", [1e295, np.inf, -np.inf])
def test_grid_overflow_is_reported(far):
    cells = patch(300, 63)
    cells[5, 2] = far
    sim = abm_b200.Simulation(cap_cells=300, jkr_table=JKR)
    sim.upload_cells(cells)
    with pytest.raises(RuntimeError, match="ABM_ERR_CAPACITY.*grid"):
        sim.get_cell_neighbors()
    sim.close()
