"""The oracle's phenotype switching and what it drives (switch.hpp:45-142; simulation.hpp:1340-1371,
1650-1656, 1831-1856, 1866-2022): Markov and inherited switching between two groups, the ramps
of switched attributes and of the adhesion energy density, the local-viscosity modulation by
group-1 contacts, and basal-only compaction.  The reference has no test of these, and its
draws come from mt19937, which the oracle replaces by its Philox policy; so the restatement is
held to statistics and closed forms:

  * Markov: a fraction dt * rate of the cells switches (within five binomial standard
    deviations), and each switched cell draws its growth rate from its new group;
  * inherit: a fraction 1 - P(g, g) of the daughter pairs switches, exactly one daughter per pair,
    either daughter equally often;
  * ramps move by |target1 - target2| / timescale per unit time (max_gamma / timescale for
    gamma) and stop at the target, at once with a zero timescale;
  * viscosity: vmin + share (vmax - vmin), the share of group-1 contacts over at least
    max_coordination_number, saturating at that many;
  * basal-only: the cells whose deepest overlap exceeds the threshold stay, in order.
This is the oracle side of the switching row; no device kernel is claimed."""
import ctypes
import math

import numpy as np
import pytest

import oracle_ref as orc

R, HALF_L = 0.8, 0.5
IP = ctypes.POINTER(ctypes.c_int)


def make(cells, **kw):
    import abm_b200
    args = dict(adhesion_mode=0, no_surface=1, iter_update_neighbors=10 ** 6, growth_mean=0.0, growth_std=0.0)
    args.update(kw)
    _, p = abm_b200.make_params(**args)
    o = orc.Oracle(p)
    o.set_cells(cells)
    return o


def switching(o, mode=1, rates=(0, 0, 0, 0), growth=((1.0, 1.5), (0.05, 0.1)), timescale=0.0, attrs=(),
              max_gamma=0.0, modulate=0, visc=(0, 0, 0, 0), max_coord=1, n_start=0):
    cols = (ctypes.c_int * 4)(*[c for c, _, _ in attrs])
    targets = np.array([t1 for _, t1, _ in attrs] + [t2 for _, _, t2 in attrs] + [0.0])
    rc = orc.LIB.oracle_set_switching(o._c, mode, n_start, orc._dp(np.array(rates, float)),
                                      orc._dp(np.array(growth[0], float)), orc._dp(np.array(growth[1], float)),
                                      timescale, len(attrs), cols, orc._dp(targets), max_gamma, modulate,
                                      orc._dp(np.array(visc, float)), max_coord)
    assert rc == 0


def colony(n, group=1, z=5.0, spacing=3.0, ncols=22):
    cells = np.zeros((n, ncols))
    side = int(math.ceil(math.sqrt(n)))
    cells[:, 0] = np.arange(n)
    cells[:, 1] = (np.arange(n) % side) * spacing
    cells[:, 2] = (np.arange(n) // side) * spacing
    cells[:, 3], cells[:, 4] = z, 1.0
    cells[:, 13], cells[:, 14] = 2 * HALF_L, HALF_L
    cells[:, 16], cells[:, 17], cells[:, 18], cells[:, 20] = 0.7, 0.072, 720.0, group
    return cells


def within(count, n, prob, k=5.0):
    return abs(count - n * prob) <= k * math.sqrt(n * prob * (1 - prob))


def test_markov_switching_statistics():
    n, rate, dt = 20000, 2.0, 0.01
    cells = colony(n)
    cells[n // 2:, 20] = 2                              # half start in group 2, which never leaves
    o = make(cells)
    switching(o, mode=1, rates=(0.0, rate, 0.0, 0.0), growth=((1.0, 1.5), (0.05, 0.1)))
    switched = orc.LIB.oracle_switch_markov(o._c, dt, 7)
    after = o.cells()
    moved = (cells[:, 20] == 1) & (after[:, 20] == 2)
    assert switched == moved.sum() and within(switched, n // 2, rate * dt)
    assert np.all(after[n // 2:, 20] == 2) and np.array_equal(after[~moved, 16], cells[~moved, 16])
    g = after[moved, 16]
    assert abs(g.mean() - 1.5) < 5 * 0.1 / math.sqrt(len(g)) and abs(g.std() - 0.1) < 0.02
    again = make(cells)
    switching(again, mode=1, rates=(0.0, rate, 0.0, 0.0), growth=((1.0, 1.5), (0.05, 0.1)))
    orc.LIB.oracle_switch_markov(again._c, dt, 7)
    assert np.array_equal(again.cells(), after)         # the same counters, the same draws
    orc.LIB.oracle_switch_markov(again._c, dt, 8)
    assert not np.array_equal(again.cells(), after)


def test_inherited_switching_statistics():
    pairs_n, stay = 20000, 0.8
    cells = colony(2 * pairs_n)
    o = make(cells)
    switching(o, mode=2, rates=(stay, 1 - stay, 0.0, 1.0), growth=((1.0, 1.5), (0.05, 0.1)))
    pairs = np.stack([np.arange(pairs_n), pairs_n + np.arange(pairs_n)], axis=1).astype(np.int32)
    switched = orc.LIB.oracle_switch_inherit(o._c, np.ascontiguousarray(pairs).ctypes.data_as(IP), pairs_n, 3)
    g = o.cells()[:, 20]
    first, second = g[:pairs_n] == 2, g[pairs_n:] == 2
    assert not np.any(first & second)                   # one daughter per pair at most
    assert switched == (first | second).sum() and within(switched, pairs_n, 1 - stay)
    assert within(first.sum(), switched, 0.5)


def test_attribute_and_gamma_ramps():
    cells = colony(4, ncols=22)
    cells[[1, 3], 20] = 2
    cells[:, 17] = 0.5                                   # ambient viscosity, the switched attribute
    cells[:, 21] = [0.0, 100.0, 40.0, 60.0]              # gamma
    o = make(cells, adhesion_mode=1)
    t1, t2, ts, gmax, dt = 0.1, 1.0, 10.0, 100.0, 1.0
    switching(o, mode=1, timescale=ts, attrs=[(17, t1, t2)], max_gamma=gmax)
    rate, grate = abs(t1 - t2) / ts, gmax / ts
    v1 = v2 = 0.5
    gam = list(cells[:, 21])
    for _ in range(12):
        orc.LIB.oracle_switch_ramps(o._c, dt)
        v1, v2 = max(v1 - rate * dt, t1), min(v2 + rate * dt, t2)
        gam = [min(gam[0] + grate * dt, gmax), max(gam[1] - grate * dt, 0.0),
               min(gam[2] + grate * dt, gmax), max(gam[3] - grate * dt, 0.0)]
        c = o.cells()
        assert abs(c[0, 17] - v1) < 1e-12 and abs(c[2, 17] - v1) < 1e-12
        assert abs(c[1, 17] - v2) < 1e-12 and abs(c[3, 17] - v2) < 1e-12
        np.testing.assert_allclose(c[:, 21], gam, atol=1e-12)
    assert c[0, 17] == t1 and c[1, 17] == t2 and c[0, 21] == gmax and c[1, 21] == 0.0
    snap = make(cells, adhesion_mode=1)
    switching(snap, mode=1, timescale=0.0, attrs=[(17, t1, t2)], max_gamma=gmax)
    orc.LIB.oracle_switch_ramps(snap._c, 1e-6)
    c = snap.cells()
    assert list(c[:, 17]) == [t1, t2, t1, t2] and list(c[:, 21]) == [gmax, 0.0, gmax, 0.0]


@pytest.mark.parametrize("max_coord", [4, 2])
def test_viscosity_follows_group_one_contacts(max_coord):
    z = 5.0
    cells = colony(5, ncols=22)
    cells[:, 1:4] = [[0, 0, z], [0, 1.5, z], [0, -1.5, z], [2 * HALF_L + 1.5, 0, z], [20, 20, z]]
    cells[:, 20] = [2, 1, 1, 2, 1]                       # the center (group 2) touches two group-1 cells
    o = make(cells, adhesion_mode=1)
    visc = (0.1, 0.3, 1.0, 5.0)                          # group 1 (min, max), group 2 (min, max)
    switching(o, mode=1, max_gamma=0.0, modulate=1, visc=visc, max_coord=max_coord)
    o.build_neighbors()
    orc.LIB.oracle_switch_ramps(o._c, 1e-3)
    eta = o.cells()[:, 17]
    share = 1.0 if 2 >= max_coord else 2 / max(3, max_coord)
    assert abs(eta[0] - (1.0 + share * 4.0)) < 1e-12
    assert eta[1] == 0.1 and eta[2] == 0.1 and eta[4] == 0.1    # no group-1 contacts
    assert eta[3] == (5.0 if max_coord == 1 else 1.0)            # touches only the group-2 center


def test_basal_only_compaction():
    cells = colony(6, z=R)
    cells[:, 4:7] = [1.0, 0.0, 0.0]
    cells[:, 3] = [0.5, 0.79, 0.81, 1.2, 0.6, 3.0]       # overlaps R - rz: 0.3, 0.01, -0.01, -0.4, 0.2, -2.2
    o = make(cells, no_surface=0)
    orc.LIB.oracle_set_basal(o._c, 1, 0.005)
    assert orc.LIB.oracle_basal_compact(o._c) == 3
    assert list(o.cells()[:, 0]) == [0, 1, 4]
    loop = make(cells, no_surface=0, max_stepsize=1e-7)
    orc.LIB.oracle_set_basal(loop._c, 1, 0.005)
    loop.loop_init()
    loop.iterate(1)
    assert list(loop.cells()[:, 0]) == [0, 1, 4] and loop.stats()["rebuilds"] >= 2


def test_switching_inside_the_loop():
    cells = colony(400, spacing=1.7)
    o = make(cells, max_stepsize=1e-5, adhesion_mode=1)
    cells[:, 21] = 0.0
    switching(o, mode=1, rates=(0.0, 2e4, 0.0, 0.0), timescale=1.0, attrs=[(17, 0.072, 0.5)], max_gamma=50.0)
    o.set_jkr_table(*orc.jkr_table(R, 0.5, 3900.0, 50.0))
    o.loop_init()
    o.iterate(5)
    c = o.cells()
    g2 = c[:, 20] == 2
    assert 0 < g2.sum() < len(c)                        # 2e4 per unit time over 5e-5: about 63%
    assert np.all(c[g2, 17] > 0.072) and np.all(c[~g2, 17] == 0.072)
    assert np.all(c[~g2, 21] > 0) and np.all(c[g2, 21] < 50.0)


def variable_table(max_gamma, nd=100, ng=50):
    d, g, r = np.zeros(nd), np.zeros(ng), np.zeros(nd * ng)
    orc.LIB.oracle_jkr_table2(R, 0.5, 3900.0, max_gamma, nd, ng, orc._dp(d), orc._dp(g), orc._dp(r))
    return d, g, r


def pair_forces(gamma, fixed=None, variable=None):
    cells = colony(2, ncols=22)
    cells[:, 1:7] = [[0, 0, 5, 1, 0, 0], [0, 1.45, 5, 1, 0, 0]]    # overlap 0.15
    cells[:, 21] = gamma
    o = make(cells, adhesion_mode=1)
    if fixed is not None:
        o.set_jkr_table(*fixed)
    else:
        d, g, r = variable
        orc.LIB.oracle_set_jkr_table2(o._c, orc._dp(d), len(d), orc._dp(g), len(g), orc._dp(r))
    o.build_neighbors()
    return o.cell_cell_forces()


def test_variable_gamma_jkr_table():
    """IsotropicJKRDataVariableGamma (mechanics.hpp:159-199, adhesion.hpp:412-526), the table the
    driver builds when switching ramps gamma (simulation.hpp:1379-1395): radii on
    LinSpaced(overlap) x LinSpaced(0, max_gamma), interpolated bilinearly.  Its gamma = 0
    column is the Hertz radius sqrt(Req delta), its last column the fixed-gamma table at
    max_gamma; the pair forces it gives equal the fixed table's at a mesh gamma and differ by
    the interpolation in gamma between mesh points (4e-4 at gamma = 37.3 with 50 points up to
    100; near gamma = 0, where the radius grows like gamma^(1/3), the reference's table is
    coarser: 10 % at gamma = 0.5)."""
    d, g, r = variable_table(100.0)
    r2 = r.reshape(len(d), len(g))
    np.testing.assert_allclose(r2[:, 0], np.sqrt(R / 2 * d), rtol=1e-14, atol=1e-15)
    df, rf = orc.jkr_table(R, 0.5, 3900.0, 100.0)
    assert np.array_equal(d, df) and np.array_equal(r2[:, -1], rf)
    for gamma in (100.0, g[2], g[25]):
        fv = pair_forces(gamma, variable=(d, g, r))
        ff = pair_forces(gamma, fixed=orc.jkr_table(R, 0.5, 3900.0, gamma))
        assert np.abs(fv - ff).max() <= 1e-13 * np.abs(ff).max(), gamma
    fv = pair_forces(37.3, variable=(d, g, r))
    ff = pair_forces(37.3, fixed=orc.jkr_table(R, 0.5, 3900.0, 37.3))
    rel = np.abs(fv - ff).max() / np.abs(ff).max()
    assert 1e-6 < rel < 1e-3, rel


def test_inherited_switching_at_division_inside_the_loop():
    """simulation.hpp:1617-1656: cells past Ldiv divide, and with P(stay) = 0 every pair of
    daughters (the mother's row, the appended row) ends with exactly one daughter in group 2."""
    import abm_b200
    n = 16
    cells = colony(n, spacing=9.0)
    _, p = abm_b200.make_params(adhesion_mode=0, no_surface=1, max_stepsize=1e-6, growth_mean=0.7,
                                growth_std=0.0, iter_update_neighbors=10 ** 6)
    cells[:, 13] = p["Ldiv"] + 0.05
    cells[:, 14] = cells[:, 13] / 2
    o = orc.Oracle(p)
    o.set_cells(cells)
    o.set_parents(np.full(n, -1, dtype=np.int32))
    switching(o, mode=2, rates=(0.0, 1.0, 0.0, 1.0), growth=((0.7, 1.4), (0.0, 0.0)))
    o.loop_init()
    o.iterate(1)
    c = o.cells()
    assert len(c) == 2 * n
    g2 = c[:, 20] == 2
    assert g2.sum() == n and np.all(g2[:n] ^ g2[n:])     # one daughter of each pair
    assert np.all(c[g2, 16] == 1.4) and np.all(c[~g2, 16] == 0.7)
