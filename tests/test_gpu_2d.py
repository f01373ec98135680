"""Parity of the 2-D CUDA path (ABM-2d) with the 2-D oracle through the C ABI.

Bars, as for 3-D: the neighbor pair set, its (d, s, t), the adhesion flags and
division events bit for bit; forces, velocities, RK states and error norms within
1e-10 normwise per column."""
import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-10
ADH = dict(adhesion_mode=1, adhesion_strength=20.0, adhesion_mindist=1.2)


def colwise_relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = np.abs(b).max(axis=0)
    diff = np.abs(a - b).max(axis=0)
    return float(np.max(np.where(scale > 0, diff / np.where(scale > 0, scale, 1), diff)))


def make_pair(cells, **kw):
    p = dict(abm_b200.DEFAULTS_2D)
    p.update(kw)
    p.setdefault("cap_cells", max(len(cells), 1) + 16)
    sim = abm_b200.Simulation(**p)
    sim.upload_cells(cells)
    o = orc.Oracle2D(sim.pdict)
    o.set_cells(cells)
    return sim, o


def colony(n, seed, **kw):
    return workloads.biofilm_2d(n, seed=seed, **kw)


@pytest.mark.parametrize("adh", [0, 1])
def test_2d_neighbor_table_and_flags_bit_exact(adh):
    cells = colony(3000, 1)
    sim, o = make_pair(cells, **(ADH if adh else {}))
    m = sim.get_cell_neighbors()
    assert m == o.build_neighbors()
    g = sim.neighbors()
    ref, flags = o.neighbors(with_adhere=True)
    assert g.shape == ref.shape == (m, 6)
    assert np.array_equal(g, ref)
    if adh:
        assert np.array_equal(sim.adhesion_flags(), flags)
        assert flags.sum() > 0


@pytest.mark.parametrize("adh", [0, 1])
def test_2d_forces_and_velocities(adh):
    cells = colony(4000, 2)
    sim, o = make_pair(cells, **(ADH if adh else {}))
    sim.get_cell_neighbors()
    o.build_neighbors()
    assert colwise_relerr(sim.cell_cell_forces(), o.cell_cell_forces()) <= RTOL
    assert colwise_relerr(sim.get_velocities(), o.get_velocities()) <= RTOL


@pytest.mark.parametrize("mode", [1, 2])
def test_2d_rk_attempt(mode):
    cells = colony(3000, 3)
    sim, o = make_pair(cells, integration_mode=mode, **ADH)
    sim.get_cell_neighbors()
    o.build_neighbors()
    for dt in (1e-5, 1e-3):
        cg, eg, mg = sim.step_runge_kutta_adaptive(dt)
        co, eo, mo = o.rk_attempt(dt)
        assert colwise_relerr(cg, co) <= RTOL
        inc = dt * np.abs(co[:, 5:9]).max(axis=0)
        assert np.all(np.abs(eg - eo).max(axis=0) <= RTOL * inc)
        y0 = cells[:, 1:5]
        assert abs(mg - mo) <= RTOL * (inc / (1e-8 * (1 + np.abs(y0)))).max()


def test_2d_rk_attempt_with_noise():
    cells = colony(2000, 4)
    sim, o = make_pair(cells, max_noise=5.0)
    sim.get_cell_neighbors()
    o.build_neighbors()
    cg, _, _ = sim.step_runge_kutta_adaptive(1e-4, attempt=2)
    co, _, _ = o.rk_attempt(1e-4, 0, 2)
    assert colwise_relerr(cg, co) <= RTOL


@pytest.mark.parametrize("graphs", [1, 0])
def test_2d_iterations_match_oracle(graphs):
    cells = colony(2000, 5)
    sim, o = make_pair(cells, use_graphs=graphs, iter_update_neighbors=10, max_stepsize=1e-3, **ADH)
    sim.get_cell_neighbors()
    o.loop_init()
    for _ in range(3):
        s = sim.iterate(12)
        o.iterate(12)
        t, dt, it = sim.clock()
        to, dto, ito = o.clock()
        assert it == ito
        assert abs(t - to) <= 1e-10 * to and abs(dt - dto) <= 1e-10 * dto
        assert colwise_relerr(sim.download_cells(), o.cells()) <= 1e-9
        assert s["attempts"] == o.stats()["attempts"]
        assert np.array_equal(sim.neighbors()[:, :2], o.neighbors()[:, :2])


DIV2 = dict(growth_mean=1.5, growth_std=0.1, daughter_length_std=0.05, daughter_angle_xy_bound=0.3, rng_seed=9,
            Ldiv=4.4, neighbor_threshold=3.2)


def test_2d_division_matches_oracle():
    cells = colony(800, 6, lmax=4.0)
    n = len(cells)
    rng = np.random.default_rng(6)
    idx = rng.choice(n, 50, replace=False)
    cells[idx, 9] = 4.5
    cells[idx, 10] = 2.25
    cells[:, 12] = rng.normal(1.5, 0.1, size=n)
    sim, o = make_pair(cells, cap_cells=2 * n, **DIV2)
    parents = -np.ones(n, dtype=np.int32)
    sim.set_parents(parents)
    o.set_parents(parents)
    sim.set_clock(0.5, 1e-5, 11)
    o.set_clock(0.5, 1e-5, 11)
    nd = sim.divide_cells()
    nd_o, tries_o = o.divide(0.5, 11)
    assert nd == nd_o == 50
    assert sim.last_division_tries() == tries_o
    cg, co = sim.download_cells(), o.cells()
    assert cg.shape == co.shape == (n + nd, workloads.NCOLS_2D)
    assert np.array_equal(sim.parents(), o.parents())
    assert np.array_equal(cg, co)                               # daughters bit for bit


@pytest.mark.parametrize("graphs", [1, 0])
def test_2d_growth_and_division_loop(graphs):
    # per-step parity from identical inputs (cells, neighbor table, adhesion flags,
    # clock, lineage), as the 3-D loop test
    cells = colony(500, 7, lmax=4.0)
    rng = np.random.default_rng(7)
    cells[:, 9] = rng.uniform(3.0, 4.35, size=len(cells))
    cells[:40, 9] = 4.4 - rng.uniform(0.0, 2e-3, size=40)
    cells[:, 10] = cells[:, 9] / 2
    cells[:, 12] = rng.normal(1.5, 0.1, size=len(cells))
    n = len(cells)
    sim, o = make_pair(cells, cap_cells=3 * n, use_graphs=graphs, max_stepsize=1e-3, iter_update_neighbors=7,
                       **DIV2, **ADH)
    o.set_parents(-np.ones(n, dtype=np.int32))
    o.loop_init()
    divided = 0
    for it in range(24):
        sim.upload_cells(o.cells())
        nb, flags = o.neighbors(with_adhere=True)
        sim.set_neighbors(nb)
        sim.set_adhesion_flags(flags)
        sim.set_clock(*o.clock())
        sim.set_parents(o.parents())
        n0 = o.cells().shape[0]
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        assert cg.shape == co.shape
        divided += co.shape[0] - n0
        assert np.array_equal(cg[:, 0], co[:, 0])
        assert np.array_equal(sim.parents(), o.parents())
        assert colwise_relerr(cg, co) <= 1e-9
        t, dt, i = sim.clock()
        to, dto, io = o.clock()
        assert i == io and abs(dt - dto) <= 1e-10 * dto
        if i % 7 == 0 or co.shape[0] != n0:
            assert np.array_equal(sim.neighbors()[:, :2], o.neighbors()[:, :2])
            assert np.array_equal(sim.adhesion_flags(), o.neighbors(with_adhere=True)[1])
    assert divided > 0


def test_2d_founder_grows_to_1000_cells():
    """The 2-D driver's run (one founder at the origin along (1, 0), L0 = 2, growth
    N(1.5, 0.1^2), Ldiv 4.4, BS32, tol 1e-8) to 1000 cells on the device."""
    sim = abm_b200.Simulation(cap_cells=1200, max_stepsize=1e-4, **dict(abm_b200.DEFAULTS_2D, **DIV2))
    sim.upload_cells(workloads.founder_2d())
    sim.set_parents([-1])
    sim.set_clock(0.0, 1e-4, 0)
    sim.get_cell_neighbors()
    st = sim.iterate(500000, n_cells_stop=1000)
    cells = sim.download_cells()
    assert cells.shape[0] >= 1000
    assert np.all(np.isfinite(cells))
    np.testing.assert_allclose(np.hypot(cells[:, 3], cells[:, 4]), 1.0, atol=1e-12)
    assert len(np.unique(cells[:, 0])) == cells.shape[0]           # distinct IDs
    # every division gives the mother's row and the new row fresh IDs: 2 n - 1 IDs from one founder
    assert len(sim.parents()) == 2 * cells.shape[0] - 1
    print("\nfounder -> %d cells: %d iterations, t = %.3f h, %d attempts" % (
        cells.shape[0], st["iterations"], st["t"], st["attempts"]))
