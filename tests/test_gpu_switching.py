"""Phenotype switching, the attribute and gamma ramps, local viscosity and basal-only
compaction on the device (switch.hpp:45-142; simulation.hpp:1650-1656, 1831-1856,
1866-2022; growth.hpp:634-644), against the oracle's restatement, through the C ABI.

Both sides draw from the same counter-based Philox policy (purpose SWITCH, counters
iteration, cell or division pair, slot), so the comparison is decision for decision, not
statistical.  Bars:
  * groups, the growth rates drawn at a switch, the IDs and the rows kept by basal-only
    compaction: bit for bit;
  * local viscosity eta0: bit for bit (integer contact counts, correctly rounded
    arithmetic) from identical inputs;
  * ramped attributes and gamma: 1e-12 relative, dt and the clock 1e-10 (the ramps advance
    by rate x dt, and dt is set by the error norm, which the device sums in another order);
  * the other columns: 1e-9 normwise, the loop tests' bar.
"""
import numpy as np
import pytest

import abm_b200
import oracle_ref as orc
from test_gpu_parity import colwise_relerr, patch_state

pytestmark = pytest.mark.gpu

MAX_GAMMA = 60.0
VTABLE = None


def vtable():
    global VTABLE
    if VTABLE is None:
        VTABLE = abm_b200.jkr_radius_table_variable(0.8, 0.5, 3900.0, MAX_GAMMA, 100, 40)
    return VTABLE


def pair(cells, switching=None, basal=None, variable=True, **kw):
    kw.setdefault("cap_cells", 3 * max(len(cells), 1) + 16)
    sim = abm_b200.Simulation(jkr_table=orc.jkr_table(0.8, 0.5, 3900.0, MAX_GAMMA), **kw)
    o = orc.Oracle(sim.pdict, jkr=orc.jkr_table(0.8, 0.5, 3900.0, MAX_GAMMA))
    if variable:
        sim.set_jkr_table_variable(*vtable())
        o.set_jkr_table_variable(*vtable())
    if switching is not None:
        sim.set_switching(**switching)
        o.set_switching(**switching)
    if basal is not None:
        sim.set_basal_only(True, basal)
        o.set_basal_only(True, basal)
    sim.upload_cells(cells)
    o.set_cells(cells)
    sim.set_parents(-np.ones(len(cells), dtype=np.int32))
    o.set_parents(-np.ones(len(cells), dtype=np.int32))
    return sim, o


def compare(cg, co, ramped=(), exact=(0, 20)):
    assert cg.shape == co.shape
    for c in exact:
        assert np.array_equal(cg[:, c], co[:, c]), c
    for c in ramped:
        scale = max(np.abs(co[:, c]).max(), 1e-300)
        assert np.abs(cg[:, c] - co[:, c]).max() <= 1e-12 * scale, c
    assert colwise_relerr(cg, co) <= 1e-9


def markov_cells(n=800, seed=61):
    cells = patch_state(n, seed)
    cells[:, 20] = 1.0
    cells[:, 21] = 10.0
    cells[: n // 3, 20] = 2.0
    cells[:, 16] = 0.0
    return cells


MARKOV = dict(mode=1, rates=(0.0, 2e4, 1e4, 0.0), growth=((0.0, 0.0), (0.0, 0.0)), timescale=2e-4,
              attrs=[(17, 100.0, 300.0), (19, 100.0, 40.0)], max_gamma=MAX_GAMMA)


@pytest.mark.parametrize("graphs", [1, 0])
def test_markov_switching_and_ramps_follow_the_oracle(graphs):
    """Twelve free-running iterations at dt <= 1e-5 h: about a fifth of the cells switch each
    iteration; every switch, ramp and clock step is the oracle's."""
    cells = markov_cells()
    sim, o = pair(cells, switching=MARKOV, max_stepsize=1e-5, iter_update_neighbors=5, use_graphs=graphs)
    sim.get_cell_neighbors()
    o.loop_init()
    switched = 0
    prev = cells[:, 20].copy()
    for it in range(12):
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        compare(cg, co, ramped=(17, 19, 21))
        switched += int((co[:, 20] != prev).sum())
        prev = co[:, 20].copy()
        t, dt, i = sim.clock()
        to, dto, io = o.clock()
        assert i == io and abs(dt - dto) <= 1e-10 * dto and abs(t - to) <= 1e-10 * to
    assert switched > len(cells)                     # many switches, both ways
    g1 = cg[:, 20] == 1
    assert 0 < g1.sum() < len(cg)
    # the ramps moved gamma off its start, within [0, max_gamma]
    assert np.count_nonzero(cg[:, 21] != 10.0) > len(cg) // 2
    assert cg[:, 21].min() >= 0.0 and cg[:, 21].max() <= MAX_GAMMA
    sim.close()


def test_markov_growth_draws_from_the_new_group():
    """A switch draws the new group's growth rate (switch.hpp:76-80); with every cell leaving
    group 1 at once (rate x dt > 1) all growth rates are group 2's draws."""
    cells = markov_cells(400, 62)
    cells[:, 20] = 1.0
    sw = dict(mode=1, rates=(0.0, 1e7, 0.0, 0.0), growth=((0.2, 1.1), (0.0, 0.05)), max_gamma=0.0)
    sim, o = pair(cells, switching=sw, max_stepsize=1e-6, iter_update_neighbors=5)
    sim.get_cell_neighbors()
    o.loop_init()
    sim.iterate(1)
    o.iterate(1)
    cg, co = sim.download_cells(), o.cells()
    assert np.all(cg[:, 20] == 2)
    compare(cg, co, exact=(0, 16, 20))
    assert abs(cg[:, 16].mean() - 1.1) < 0.02 and 0.03 < cg[:, 16].std() < 0.07
    sim.close()


def test_switching_starts_at_n_start():
    cells = markov_cells(400, 63)
    sw = dict(MARKOV, n_start=401)
    sim, o = pair(cells, switching=sw, max_stepsize=1e-5)
    sim.get_cell_neighbors()
    o.loop_init()
    sim.iterate(3)
    o.iterate(3)
    cg, co = sim.download_cells(), o.cells()
    assert np.array_equal(cg[:, 20], cells[:, 20])   # no cell switched below n_start
    compare(cg, co, ramped=(17, 19, 21))
    sim.close()


@pytest.mark.parametrize("timescale", [0.0, 3e-5])
def test_local_viscosity_and_gamma_ramp(timescale):
    """simulation.hpp:1940-2020 from identical inputs each iteration: eta0 from the share of
    group-1 contacts (saturating at max_coord), gamma ramped, over seven iterations that
    include a periodic rebuild."""
    cells = markov_cells(900, 64)
    sw = dict(MARKOV, timescale=timescale, modulate=1, visc=(50.0, 900.0, 20.0, 400.0), max_coord=3, attrs=[])
    sim, o = pair(cells, switching=sw, max_stepsize=1e-5, iter_update_neighbors=3)
    sim.get_cell_neighbors()
    o.loop_init()
    for it in range(7):
        sim.upload_cells(o.cells())
        sim.set_neighbors(o.neighbors())
        sim.set_clock(*o.clock())
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        compare(cg, co, ramped=(21,), exact=(0, 17, 20))
        assert np.array_equal(sim.neighbors()[:, :2], o.neighbors()[:, :2])
    eta0 = cg[:, 17]
    assert len(np.unique(eta0)) > 3 and eta0.min() >= 20.0 and eta0.max() <= 900.0
    sim.close()


def division_cells(n=64, seed=65):
    cells = patch_state(n, seed)
    rng = np.random.default_rng(seed)
    cells[:, 1:3] *= 2.5                              # room to divide
    cells[:, 13] = 5.65 + rng.uniform(0.0, 0.05, size=n)
    cells[:, 14] = cells[:, 13] / 2
    cells[:, 16] = 0.7
    cells[:, 20] = 1.0
    cells[: n // 4, 20] = 2.0
    return cells


@pytest.mark.parametrize("stay", [0.0, 0.5])
def test_inherited_switching_at_division(stay):
    """switch.hpp:97-142 at simulation.hpp:1650-1656: each pair of daughters (the mother's row,
    the appended row); with P(stay) = 0 exactly one daughter of every pair changes group and
    draws that group's growth rate.  Daughters of either group draw their mother's group's
    distribution (growth.hpp:634-644)."""
    cells = division_cells()
    n = len(cells)
    sw = dict(mode=2, rates=(stay, 1.0 - stay, 0.0, 1.0), growth=((0.7, 1.4), (0.05, 0.1)))
    sim, o = pair(cells, switching=sw, variable=False, adhesion_mode=0, max_stepsize=1e-6,
                  growth_mean=0.7, growth_std=0.0)
    sim.get_cell_neighbors()
    o.loop_init()
    sim.iterate(1)
    o.iterate(1)
    cg, co = sim.download_cells(), o.cells()
    assert len(co) == 2 * n
    compare(cg, co, exact=(0, 16, 20))
    assert np.array_equal(sim.parents(), o.parents())
    moved = (cg[:n, 20] != cells[:, 20]) | (cg[n:, 20] != cells[:, 20])
    both = (cg[:n, 20] != cells[:, 20]) & (cg[n:, 20] != cells[:, 20])
    g1 = cells[:, 20] == 1
    assert not both.any() and not moved[~g1].any()      # P(2, 2) = 1: group-2 pairs stay
    if stay == 0.0:
        assert moved[g1].all()
    else:
        assert 0 < moved[g1].sum() < g1.sum()
    sim.close()


def basal_cells(n=600, seed=66):
    cells = patch_state(n, seed)
    rng = np.random.default_rng(seed)
    cells[:, 16] = rng.uniform(0.5, 1.0, size=n)
    return cells


@pytest.mark.parametrize("graphs", [1, 0])
def test_basal_only_compaction(graphs):
    """simulation.hpp:1831-1856: after each accepted step only the cells whose deepest overlap
    R - rz + half_l nz exceeds the threshold stay, in their order, and the neighbor list is
    rebuilt for them."""
    cells = basal_cells()
    sim, o = pair(cells, basal=0.01, variable=False, max_stepsize=1e-5, iter_update_neighbors=4,
                  use_graphs=graphs)
    sim.get_cell_neighbors()
    o.loop_init()
    for it in range(6):
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        compare(cg, co)
        assert np.array_equal(sim.neighbors()[:, :2], o.neighbors()[:, :2])
    assert len(co) < len(cells)
    assert sim.basal_dropped() == len(cells) - len(co)
    keep = 0.8 - co[:, 3] + co[:, 14] * co[:, 6] > 0.01
    assert keep.all()
    sim.close()


def test_switching_graph_and_stream_paths_agree():
    """The conditional-node graph and the stream path (host decisions) run the same kernels:
    the same end state bit for bit after iterations with division, inherited switching,
    periodic rebuilds and the ramps."""
    cells = division_cells(96, 67)
    cells[:, 21] = 5.0
    sw = dict(mode=2, rates=(0.5, 0.5, 0.2, 0.8), growth=((0.7, 1.4), (0.05, 0.1)), timescale=1e-4,
              attrs=[(18, 720.0, 200.0)], max_gamma=MAX_GAMMA, modulate=1, visc=(50.0, 900.0, 20.0, 400.0),
              max_coord=2)
    out = []
    for graphs in (1, 0):
        sim, _ = pair(cells, switching=sw, max_stepsize=1e-5, iter_update_neighbors=4, use_graphs=graphs,
                      growth_mean=0.7, growth_std=0.0)
        sim.get_cell_neighbors()
        sim.iterate(9)
        out.append((sim.download_cells(), sim.neighbors(), sim.clock()))
        sim.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


def test_switching_arguments_are_checked():
    cells = markov_cells(50, 68)
    sim = abm_b200.Simulation(jkr_table=orc.jkr_table(0.8, 0.5, 3900.0, MAX_GAMMA), cap_cells=64)
    sim.upload_cells(cells)
    for bad in (dict(mode=3), dict(attrs=[(16, 1.0, 2.0)]), dict(rates=(0.0, -1.0, 0.0, 0.0)),
                dict(max_coord=0), dict(timescale=-1.0)):
        with pytest.raises(RuntimeError):
            sim.set_switching(**dict(MARKOV, **bad))
    sim.close()
