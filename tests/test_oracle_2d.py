"""The 2-D oracle (oracle/abm2d.hpp) against the reference's own 2-D known-answer
cases: segment distances (2D/test/src/testDistBetweenCells.cpp, committed as
tests/golden/dist2d_cases.json), Hertz forces and torques
(2D/test/src/testHertz.cpp:370-591) and JKR-Lagrange adhesion
(2D/test/src/testAdhesion.cpp:1519-1596)."""
import json
import math
import os

import numpy as np
import pytest

import oracle_ref as orc
from abm_b200 import workloads

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden2d():
    with open(os.path.join(GOLDEN, "dist2d_cases.json")) as f:
        return json.load(f)


def z0(v):
    return [v[0], v[1], 0.0]


@pytest.mark.parametrize("k", range(16))
def test_oracle_distance_golden_2d(k):
    c = golden2d()["dist_cases"][k]
    d, s, t = orc.dist_between_cells(z0(c["r1"]), z0(c["n1"]), c["half_l1"], z0(c["r2"]), z0(c["n2"]), c["half_l2"])
    assert abs(d[2]) == 0.0
    np.testing.assert_allclose(d[:2], c["d"], atol=1e-8, rtol=0)
    assert abs(s - c["s"]) <= 1e-8 and abs(t - c["t"]) <= 1e-8


def test_oracle_nearest_golden_2d():
    for c in golden2d()["nearest_cases"]:
        assert abs(orc.nearest_body_coord(z0(c["r"]), z0(c["n"]), c["half_l"], z0(c["q"])) - c["target"]) <= 1e-8


def two_cells_2d(r1, n1, h1, r2, n2, h2):
    """The two-cell array of testHertz.cpp:196-198 (17 columns)."""
    cells = np.zeros((2, workloads.NCOLS_2D), order="F")
    for i, (r, n, h) in enumerate(((r1, n1, h1), (r2, n2, h2))):
        cells[i] = [i, r[0], r[1], n[0], n[1], 0, 0, 0, 0, 2 * h, h, 0, 1, 1, 1, 1, 1]
    return cells


SIX = math.pi / 6


def hertz_cases():
    """(r1, n1, h1, r2, n2, h2, target_force_21) of testHertz.cpp:370-591 with R = 0.8,
    Rcell = 0.5, E0 = 1, Ecell = 100."""
    R, Rcell, E0, Ecell = 0.8, 0.5, 1.0, 100.0
    hard = lambda dist: (2.5 * E0 * math.sqrt(R) * (2 * (R - Rcell)) ** 1.5
                         + 2.5 * Ecell * math.sqrt(Rcell) * (2 * Rcell - dist) ** 1.5)
    soft = lambda dist: 2.5 * E0 * math.sqrt(R) * (2 * R - dist) ** 1.5
    cases = []
    # skew cells (:370-455)
    cases.append(((2, 1), (0.6, 0.8), 1, (0, 3), (0, 1), 0.5, np.zeros(2)))
    r2 = (0.5 + 0.5 * math.cos(SIX), 1 + 0.5 * math.sin(SIX))
    n2 = (math.cos(SIX), math.sin(SIX))
    cases.append(((0, 0), (1, 0), 0.5, r2, n2, 0.5, -np.array([0.0, 1.0]) * hard(1.0)))
    r2 = (0.2 + 0.5 * math.cos(SIX), 1 + 0.5 * math.sin(SIX))
    cases.append(((0, 0), (1, 0), 0.5, r2, n2, 0.5, -np.array([0.0, 1.0]) * hard(1.0)))
    d12 = np.array([1.4 / math.sqrt(2.0), 1.4 / math.sqrt(2.0)])
    dist = np.linalg.norm(d12)
    cases.append(((0, 0), (1, 0), 0.5, (0.5 + 1.4 / math.sqrt(2.0), 1.4 / math.sqrt(2.0)),
                  (1 / math.sqrt(2.0), -1 / math.sqrt(2.0)), 0.5, -d12 / dist * soft(dist)))
    # parallel cells (:457-543)
    d12 = np.array([1.4, 0.0])
    cases.append(((0, 0), (1, 0), 0.5, (2.4, 0), (1, 0), 0.5, -d12 / 1.4 * soft(1.4)))
    d12 = np.array([1.4 * math.cos(SIX), 1.4 * math.sin(SIX)])
    dist = np.linalg.norm(d12)
    cases.append(((0, 0), (1, 0), 0.5, (1.0 + 1.4 * math.cos(SIX), 1.4 * math.sin(SIX)), (1, 0), 0.5,
                  -d12 / dist * soft(dist)))
    d12 = np.array([0.0, 1.5])
    t15 = -d12 / 1.5 * soft(1.5)
    cases.append(((0, 0), (1, 0), 0.5, (0, 1.5), (1, 0), 0.5, t15))
    cases.append(((0, 0), (1, 0), 0.5, (0.2, 1.5), (1, 0), 0.5, t15))
    cases.append(((0, 0), (1, 0), 1, (-0.3, 1.5), (1, 0), 0.5, t15))
    # perpendicular cells (:545-591)
    t_perp = -np.array([1.0, 0.0]) * hard(1.0)
    cases.append(((0, 0), (1, 0), 0.5, (1.5, 0), (0, 1), 0.5, t_perp))
    cases.append(((0, 0), (1, 0), 0.5, (1.5, 0.2), (0, 1), 0.5, t_perp))
    return cases


def cross3(a, b):
    return np.cross(np.array([a[0], a[1], 0.0]), np.array([b[0], b[1], 0.0]))


@pytest.mark.parametrize("k", range(11))
def test_oracle_hertz_known_answers_2d(k):
    r1, n1, h1, r2, n2, h2, target = hertz_cases()[k]
    R, Rcell, E0, Ecell = 0.8, 0.5, 1.0, 100.0
    # the test's own prefactors (testHertz.cpp:201-204)
    pf = (2.5 * E0 * math.sqrt(R), 2.5 * E0 * math.sqrt(R) * (2 * (R - Rcell)) ** 1.5, 2.5 * Ecell * math.sqrt(R))
    o = orc.Oracle2D(dict(R=R, Rcell=Rcell, E0=E0, Ecell=Ecell, neighbor_threshold=10.0, Ldiv=5.6,
                          adhesion_mode=0), pf=pf)
    o.set_cells(two_cells_2d(r1, n1, h1, r2, n2, h2))
    o.build_neighbors()
    nb = o.neighbors()
    dist = np.linalg.norm(nb[0, 2:4]) if len(nb) else np.inf
    thr = 1e-8 * Ecell if dist < R + Rcell else (1e-8 * E0 if dist < 2 * R else 1e-8)
    forces1 = -o.cell_cell_forces()
    # translational force on cell 0 (the rows of the reference's table are (i, j) with j < i,
    # so cell 0 is the table's "j"; the target is the force on the first cell of the test)
    assert np.linalg.norm(forces1[0, :2] - target) <= thr
    assert np.linalg.norm(forces1[0, :2] + forces1[1, :2]) <= thr
    if len(nb):
        s = nb[0, 5]                     # cell-body coordinate on cell 0 (the row's sj)
        u = np.array([n1[0], n1[1]])
        torque = np.cross(cross3(s * u, target), np.array([u[0], u[1], 0.0]))[:2]
        assert np.linalg.norm(forces1[0, 2:4] - torque) <= thr


def jkr_cases():
    """(r1, n1, h1, r2, n2, h2, target_force_21) of testAdhesion.cpp:1519-1596, R = 0.8, dmin = 1.2."""
    R, dmin = 0.8, 1.2
    r2 = (0.5 + 0.5 * math.cos(SIX), 1 + 0.5 * math.sin(SIX))
    n2 = (math.cos(SIX), math.sin(SIX))
    t_min = np.array([0.0, 1.0]) * math.pi * R * (2 * R - dmin)
    d12 = np.array([1.4 / math.sqrt(2.0), 1.4 / math.sqrt(2.0)])
    dist = np.linalg.norm(d12)
    return [((2, 1), (0.6, 0.8), 1, (0, 3), (0, 1), 0.5, np.zeros(2)),
            ((0, 0), (1, 0), 0.5, r2, n2, 0.5, t_min),
            ((0, 0), (1, 0), 0.5, (0.2 + 0.5 * math.cos(SIX), 1 + 0.5 * math.sin(SIX)), n2, 0.5, t_min),
            ((0, 0), (1, 0), 0.5, (0.5 + 1.4 / math.sqrt(2.0), 1.4 / math.sqrt(2.0)),
             (1 / math.sqrt(2.0), -1 / math.sqrt(2.0)), 0.5, d12 / dist * math.pi * R * (2 * R - dist))]


@pytest.mark.parametrize("k", range(4))
def test_oracle_jkr_lagrange_known_answers_2d(k):
    r1, n1, h1, r2, n2, h2, target = jkr_cases()[k]
    d, s, t = orc.dist_between_cells(z0(r1), z0(n1), h1, z0(r2), z0(n2), h2)
    f = -orc.jkr_lagrange_pair(n1, n2, d[:2], 0.8, s, t, 1.2)
    assert np.linalg.norm(f[0, :2] - target) <= 1e-7
    u = np.array([n1[0], n1[1]])
    torque = np.cross(cross3(s * u, target), np.array([u[0], u[1], 0.0]))[:2]
    assert np.linalg.norm(f[0, 2:4] - torque) <= 1e-7


def test_oracle_2d_isolated_cell_is_stationary_and_founder_divides():
    o = orc.Oracle2D(dict(R=0.8, Rcell=0.5, E0=3900.0, Ecell=3.9e6, Ldiv=4.4, neighbor_threshold=3.2,
                          integration_mode=2, max_stepsize=1e-3, growth_mean=1.5, growth_std=0.1,
                          daughter_length_std=0.01, daughter_angle_xy_bound=0.1))
    o.set_cells(workloads.founder_2d())
    o.set_parents([-1])
    o.loop_init()
    np.testing.assert_array_equal(o.get_velocities(), 0.0)
    o.iterate(2000)
    c = o.cells()
    assert c.shape[0] >= 2                          # the founder reached Ldiv and divided
    assert np.all(np.isfinite(c))
    np.testing.assert_allclose(np.hypot(c[:, 3], c[:, 4]), 1.0, atol=1e-12)
