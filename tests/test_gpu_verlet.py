"""Velocity Verlet on the device (integration mode 0: stepVelocityVerlet,
mechanics.hpp:2668-2996, with the include_constraint forces of mechanics.hpp:673-910,
1031-1175, 1209-1659 and adhesion.hpp:282-526, the ambient viscosity and cell-surface
friction of mechanics.hpp:1784-1917, and the driver's density, simulation.hpp:1279-1290
and 1786-1798) against the oracle's restatement, through the C ABI.

Bar: 1e-9 normwise per column after each step from the oracle's own state (the loop tests'
bar), and after several free-running steps; the pair set and the clock exactly.
"""
import numpy as np
import pytest

import abm_b200
import oracle_ref as orc
from test_gpu_parity import colwise_relerr, patch_state

pytestmark = pytest.mark.gpu

R = 0.8
JKR = orc.jkr_table(R, 0.5, 3900.0, 100.0, 100)


def moving(cells, seed, scale=0.3):
    """Give the cells stored velocities (dn perpendicular to n)."""
    rng = np.random.default_rng(seed)
    c = np.array(cells, order="F")
    c[:, 7:10] = rng.normal(0.0, scale, (len(c), 3))
    dn = rng.normal(0.0, scale, (len(c), 3))
    nn = c[:, 4:7]
    c[:, 10:13] = dn - (dn * nn).sum(1, keepdims=True) * nn
    return c


def pair(cells, **kw):
    kw.setdefault("cap_cells", 2 * len(cells) + 16)
    kw.setdefault("M0", 30.0)          # stable at dt = 1e-5 h against the l^9 rotational drag
    kw.setdefault("L0", 2.0)
    sim = abm_b200.Simulation(jkr_table=JKR, integration_mode=abm_b200.VELOCITY_VERLET, **kw)
    sim.upload_cells(cells)
    o = orc.Oracle(sim.pdict, jkr=JKR)
    o.set_cells(cells)
    return sim, o


@pytest.mark.parametrize("adhesion,no_surface", [(1, 0), (0, 0), (1, 1)])
def test_verlet_steps_from_the_oracle_state(adhesion, no_surface):
    cells = moving(patch_state(2000, 81), 81)
    sim, o = pair(cells, adhesion_mode=adhesion, no_surface=no_surface, max_stepsize=1e-5,
                  iter_update_neighbors=3, max_rxy_noise=5.0, max_rz_noise=5.0, max_nxy_noise=2.0,
                  max_nz_noise=2.0, rng_seed=4)
    sim.get_cell_neighbors()
    o.loop_init()
    for it in range(5):
        sim.upload_cells(o.cells())
        sim.set_neighbors(o.neighbors())
        sim.set_clock(*o.clock())
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        err = colwise_relerr(cg, co)
        assert err <= 1e-9, (it, err)
        t, dt, i = sim.clock()
        to, dto, io = o.clock()
        assert i == io and dt == dto and abs(t - to) <= 1e-12 * to
    # the step moved the cells: the velocities changed under the forces
    assert colwise_relerr(co[:, 7:13], cells[:, 7:13]) > 1e-3
    sim.close()


@pytest.mark.parametrize("graphs", [1, 0])
def test_verlet_free_running_loop(graphs):
    """Twelve steps with periodic rebuilds, running free: the oracle's trajectory."""
    cells = moving(patch_state(1500, 82), 82)
    sim, o = pair(cells, adhesion_mode=1, max_stepsize=1e-5, iter_update_neighbors=4, use_graphs=graphs)
    sim.get_cell_neighbors()
    o.loop_init()
    s = sim.iterate(12)
    o.iterate(12)
    assert colwise_relerr(sim.download_cells(), o.cells()) <= 1e-9
    assert np.array_equal(sim.neighbors()[:, :2], o.neighbors()[:, :2])
    assert s["attempts"] == o.stats()["attempts"] == 12
    assert s["iterations"] == 12
    sim.close()


def test_verlet_with_friction_and_planar_contacts():
    """Cell-cell friction in its include_constraint form, (s n) x F (mechanics.hpp:1152-1161)."""
    cells = moving(patch_state(1500, 83), 83)
    cells = np.hstack([cells[:, :22], np.random.default_rng(83).uniform(1.0, 8.0, (len(cells), 1))])
    cells = np.asfortranarray(cells)
    sim, o = pair(cells, adhesion_mode=1, friction_mode=1, cell_cell_coulomb_coeff=1.0, max_stepsize=1e-5)
    sim.get_cell_neighbors()
    o.loop_init()
    for it in range(4):
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        assert colwise_relerr(cg, co) <= 1e-9, it
    sim.close()


def test_verlet_growth_and_division():
    cells = moving(patch_state(300, 84), 84)
    rng = np.random.default_rng(84)
    cells[:, 1:3] *= 2.0
    cells[:30, 13] = 5.65
    cells[:, 14] = cells[:, 13] / 2
    cells[:, 16] = rng.uniform(0.5, 1.0, len(cells))
    sim, o = pair(cells, adhesion_mode=1, max_stepsize=1e-5, growth_mean=0.7)
    sim.set_parents(-np.ones(len(cells), dtype=np.int32))
    o.set_parents(-np.ones(len(cells), dtype=np.int32))
    sim.get_cell_neighbors()
    o.loop_init()
    for it in range(3):
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        assert cg.shape == co.shape and len(cg) >= len(cells) + 30
        assert colwise_relerr(cg, co) <= 1e-9, it
        assert np.array_equal(sim.parents(), o.parents())
    sim.close()


def test_verlet_arguments_are_checked():
    for bad in (dict(M0=0.0), dict(precision=abm_b200.PRECISION_MIXED), dict(controller=abm_b200.CONTROLLER_PI)):
        kw = dict(cap_cells=16, M0=1.0)
        kw.update(bad)
        with pytest.raises(RuntimeError):
            abm_b200.Simulation(jkr_table=JKR, integration_mode=abm_b200.VELOCITY_VERLET, **kw)
    sim = abm_b200.Simulation(jkr_table=JKR, integration_mode=abm_b200.VELOCITY_VERLET, cap_cells=16, M0=1.0)
    sim.upload_cells(patch_state(10, 85))
    sim.get_cell_neighbors()
    with pytest.raises(RuntimeError, match="Verlet"):
        sim.step_runge_kutta_adaptive(1e-6)
    sim.close()


def test_verlet_with_markov_switching():
    """The post-step kernels follow a Verlet step as they follow a Runge-Kutta one."""
    cells = moving(patch_state(800, 86), 86)
    cells[:, 20] = 1.0
    cells[:, 21] = 10.0
    sw = dict(mode=1, rates=(0.0, 2e4, 1e4, 0.0), growth=((0.0, 0.0), (0.0, 0.0)), timescale=2e-4,
              attrs=[(18, 720.0, 300.0)], max_gamma=60.0)
    sim, o = pair(cells, adhesion_mode=1, max_stepsize=1e-5, iter_update_neighbors=3)
    sim.set_switching(**sw)
    o.set_switching(**sw)
    sim.get_cell_neighbors()
    o.loop_init()
    for it in range(6):
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        assert np.array_equal(cg[:, 20], co[:, 20]), it
        assert colwise_relerr(cg, co) <= 1e-9, it
    assert np.count_nonzero(cg[:, 20] == 2) > 0
    sim.close()
