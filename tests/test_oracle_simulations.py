"""Whole-loop pins of the oracle (restated loop body of runSimulation, simulation.hpp:1617-1864),
from the reference's simulation tests, restated in today's column layout (indices.hpp):

  testVertical.cpp:32-237    one vertical cell, just touching the surface, pressed into
                             it, and clear of it: after the run nothing but rz has
                             changed, the cell is at rest, and rz is the JKR-like balance
                             half_l + R (1 - (3 pi sigma0 / (4 R E0))^(2/3)) (or its start
                             when clear), to 1e-8.
  testTwoCellSimulations.cpp:35-308
                             two cells with the surface switched off, in nine parallel,
                             perpendicular and skew arrangements at segment distances 1.0,
                             1.4 and 1.8: overlapping pairs are pushed out to 2R, clear
                             pairs do not move.  The reference prints these distances
                             without asserting them; here they are asserted, together with
                             the closed-form Hertz decay of the overlap for the arrangements
                             where the force stays on one line.
  testSkew.cpp:78-331        one cell tilted at ten angles, barely and deeply in contact:
                             it ends at rest, horizontal or vertical as the reference's
                             energy rule says, at the analytic height, to 1e-8; clear of
                             the surface, it stays where it is.

The reference's step caps (1e-7; 1e-6 for the tilted cell), step floors, error bound (1e-10)
and iteration counts are kept, except that the just-touching vertical cell runs 60000 iterations
instead of 10000: under the 1e-10 bound its fall from first contact takes steps of a
few 1e-9 and needs that many to settle."""
import math

import numpy as np
import pytest

import oracle_ref as orc

R, RCELL, HALF_L, E0, SIGMA0 = 0.8, 0.5, 0.5, 3900.0, 100.0


def params(**kw):
    import abm_b200
    args = dict(adhesion_mode=0, max_stepsize=1e-7, min_stepsize=1e-9, max_error_allowed=1e-10,
                min_error=1e-30, max_tries_update_stepsize=3, iter_update_stepsize=1,
                iter_update_neighbors=100, nz_threshold=1e-20, cell_surface_coulomb_coeff=0.0,
                L0=2 * HALF_L, Ldiv=2 * (R + 2 * HALF_L), neighbor_threshold=2 * (2 * R + 2 * HALF_L),
                Rcell=RCELL, E0=E0, Ecell=3900000.0, growth_mean=0.0, growth_std=0.0)
    args.update(kw)
    _, p = abm_b200.make_params(**args)
    return p


def run(p, cells, iters):
    o = orc.Oracle(p)
    o.set_cells(cells)
    o.loop_init()
    o.iterate(iters)
    return o.cells(), o.clock()


def cell_row(r, n, eta0):
    row = np.zeros(21)
    row[1:4], row[4:7] = r, n
    row[13], row[14] = 2 * HALF_L, HALF_L
    row[17], row[18], row[19], row[20] = eta0, 720.0, SIGMA0, 1
    return row


@pytest.mark.parametrize("start, iters", [(0.999, 60000), (0.8, 10000), (1.1, 10000)],
                         ids=["touching", "pressed", "clear"])
def test_vertical_cell(start, iters):
    z0 = HALF_L + start * R
    before = cell_row((0.0, 0.0, z0), (0.0, 0.0, 1.0), 0.072)[None, :]
    after, _ = run(params(), before, iters)
    delta = 1e-8                                       # testVertical.cpp:106
    unchanged = [c for c in range(21) if c not in (3, 7, 8, 9, 10, 11, 12)]
    assert np.all(np.abs(after[0, unchanged] - before[0, unchanged]) < delta)
    assert np.all(np.abs(after[0, 7:13]) < delta)      # at rest
    target = z0 if start > 1 else HALF_L + R * (1 - (0.75 * math.pi * SIGMA0 / (R * E0)) ** (2.0 / 3.0))
    assert abs(after[0, 3] - target) < delta, (after[0, 3], target)


C30, S30 = math.cos(math.pi / 6), math.sin(math.pi / 6)
Z = 1.1 * R
X, Y, SKEW = (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (C30, S30, 0.0)
# second cell (center, orientation) at segment distance d from the first, which sits at
# (0, 0, 1.1 R) along x (testTwoCellSimulations.cpp:139-306); True where the force stays
# on the line between the centers, so the overlap obeys d(delta)/dt = -2 F(delta) / (eta0 l)
ARRANGEMENTS = {
    "head-to-head": (lambda d: ((2 * HALF_L + d, 0, Z), X), True),
    "side-by-side": (lambda d: ((0, d, Z), X), True),
    "shifted side-by-side": (lambda d: ((0.2, d, Z), X), False),
    "T": (lambda d: ((HALF_L + d, 0, Z), Y), True),
    "shifted T": (lambda d: ((HALF_L + d, 0.2, Z), Y), False),
    "cross": (lambda d: ((0, 0, Z + d), Y), True),
    "skew end-to-end": (lambda d: ((HALF_L + d + HALF_L * C30, HALF_L * S30, Z), SKEW), False),
    "skew side-by-side": (lambda d: ((HALF_L * C30, d + HALF_L * S30, Z), SKEW), False),
    "skew cross": (lambda d: ((0.2, 0, Z + d), SKEW), False),
}


def distance(cells):
    v, _, _ = orc.dist_between_cells(cells[0, 1:4], cells[0, 4:7], HALF_L, cells[1, 1:4], cells[1, 4:7], HALF_L)
    return float(np.linalg.norm(v))


@pytest.mark.parametrize("d", [1.0, 1.4, 1.8])
def test_two_cell_simulations(d):
    eta0 = 1e-3
    p = params(no_surface=1)
    for name, (place, on_line) in ARRANGEMENTS.items():
        r2, n2 = place(d)
        cells = np.stack([cell_row((0.0, 0.0, Z), X, eta0), cell_row(r2, n2, eta0)])
        cells[1, 0] = 1
        assert abs(distance(cells) - d) < 1e-12, name
        after, (t, _, _) = run(p, cells, 10000)
        dist = distance(after)
        if d >= 2 * R:                                 # clear of each other: nothing moves
            assert np.array_equal(after[:, 1:7], cells[:, 1:7]), name
            continue
        assert 2 * R - 2e-7 < dist <= 2 * R, (name, dist)
        # overlap at most 2 (R - Rcell) throughout: the E0 Hertz law alone (mechanics.hpp:1263-1277)
        if on_line and 2 * R - d <= 2 * (R - RCELL) + 1e-12:
            k = 2 * (4.0 / 3.0) * E0 * math.sqrt(R / 2) / (eta0 * 2 * HALF_L)
            expect = ((2 * R - d) ** -0.5 + 0.5 * k * t) ** -2
            assert abs((2 * R - dist) - expect) < 1e-2 * expect, (name, 2 * R - dist, expect)


def more_adhesive_than_repulsive(rz, nz):
    """testSkew.cpp:46-73 (moreAdhesiveThanRepulsive), the reference's rule for which way a tilted
    cell ends: the adhesion energy -sigma0 areaIntegral1 against the repulsion energy."""
    if nz > 1e-20:
        ss = (R - rz) / nz
        i1 = orc.LIB.oracle_integral1(rz, nz, R, HALF_L, 2.0, ss)
        i2 = orc.LIB.oracle_integral1(rz, nz, R, HALF_L, 1.5, ss)
        e_rep = E0 * math.sqrt(R) * (R ** -0.5 * (1 - nz * nz) * i1 + 4.0 / 3.0 * nz * nz * i2)
        area = np.zeros(3)
        orc.LIB.oracle_area_integrals(rz, nz, R, HALF_L, area.ctypes.data_as(orc.ctypes.POINTER(orc.ctypes.c_double)))
        return -SIGMA0 * area[0] >= e_rep
    return rz >= R * (1 - (0.25 * SIGMA0 / (R * E0)) ** (2.0 / 3.0))


@pytest.mark.parametrize("i", range(10))
def test_skew_cell(i):
    """testSkew.cpp:78-331: a cell tilted at pi/2 (i + 1)/10, overlapping the surface by 0.001 R
    and by 0.2 R at its lower end, ends at rest either horizontal at R (1 - (sigma0/(4 R E0))^(2/3))
    or vertical at half_l + R (1 - (3 pi sigma0/(4 R E0))^(2/3)), as the reference's rule says,
    to 1e-8; 0.01 R clear of the surface, it does not move.  The reference runs up to 1e6 iterations at steps of at most 1e-6; the run here
    stops once every velocity is below 1e-9, within the same budget."""
    p = params(max_stepsize=1e-6, min_stepsize=1e-8)
    angle = math.pi / 2 * (i + 1) / 10
    for max_overlap in (0.001 * R, 0.2 * R, -0.01 * R):
        rz = R + HALF_L * math.sin(angle) - max_overlap
        before = cell_row((0.0, 0.0, rz), (math.cos(angle), 0.0, math.sin(angle)), 0.072)[None, :]
        o = orc.Oracle(p)
        o.set_cells(before)
        o.loop_init()
        for _ in range(100):
            o.iterate(10000)
            after = o.cells()
            if np.abs(after[0, 7:13]).max() < 1e-9:
                break
        delta = 1e-8                                   # testSkew.cpp:162
        assert np.all(np.abs(after[0, 7:13]) < delta), (i, max_overlap)
        kept = [0, 5] + list(range(13, 21))            # ID, ny, lengths, birth, growth, viscosities, sigma0, group
        assert np.all(np.abs(after[0, kept] - before[0, kept]) < delta)
        if max_overlap < 0:                            # clear of the surface: nothing moves
            n_end, z_end = tuple(before[0, 4:7]), rz
        elif more_adhesive_than_repulsive(rz, math.sin(angle)):
            n_end, z_end = (1.0, 0.0, 0.0), R * (1 - (0.25 * SIGMA0 / (R * E0)) ** (2.0 / 3.0))
        else:
            n_end, z_end = (0.0, 0.0, 1.0), HALF_L + R * (1 - (0.75 * math.pi * SIGMA0 / (R * E0)) ** (2.0 / 3.0))
        assert np.all(np.abs(after[0, 4:7] - n_end) < delta), (i, max_overlap, after[0, 4:7])
        assert abs(after[0, 3] - z_end) < delta, (i, max_overlap, after[0, 3], z_end)
