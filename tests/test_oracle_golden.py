"""The oracle checked against the reference's own known-answer cases and invariants.

Golden vectors: tests/golden/dist3d_cases.json, extracted by make_golden.py
from ABM-3d/ABM-3d-cpp/test/src/testDistBetweenCells.cpp (tolerance 1e-8,
as asserted there).  JKR invariants: testJKR.cpp:26-83; JKR radius against the
closed form: testContactArea.cpp:102-161.  Single-cell
stationarity: testHorizontal.cpp:79-126.  Velocity identity M v = F + 2 lambda n:
testVelocities.cpp:40-131.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle_ref as orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden(dim):
    with open(os.path.join(GOLDEN, "dist%dd_cases.json" % dim)) as f:
        return json.load(f)


def test_golden_file_counts():
    g = _golden(3)
    # testDistBetweenCells.cpp: 9 skew + 11 parallel distBetweenCells cases, 3 nearest-point cases
    assert len(g["dist_cases"]) == 20
    assert len(g["nearest_cases"]) == 3


@pytest.mark.parametrize("k", range(20))
def test_oracle_distance_golden_3d(k):
    c = _golden(3)["dist_cases"][k]
    d, s, t = orc.dist_between_cells(c["r1"], c["n1"], c["half_l1"], c["r2"], c["n2"], c["half_l2"])
    tol = 1e-8
    np.testing.assert_allclose(d, c["d"], atol=tol, rtol=0)
    assert abs(s - c["s"]) <= tol and abs(t - c["t"]) <= tol


def test_oracle_nearest_golden_3d():
    for c in _golden(3)["nearest_cases"]:
        s = orc.nearest_body_coord(c["r"], c["n"], c["half_l"], c["q"])
        assert abs(s - c["target"]) <= 1e-8


def test_oracle_distance_symmetry_random():
    # swapping the cells swaps (s, t) and negates d for skew configurations
    rng = np.random.default_rng(3)
    for _ in range(200):
        r1, r2 = rng.normal(size=3) * 2, rng.normal(size=3) * 2
        n1, n2 = rng.normal(size=3), rng.normal(size=3)
        n1 /= np.linalg.norm(n1)
        n2 /= np.linalg.norm(n2)
        if abs(n1 @ n2) >= 0.9999:
            continue
        h1, h2 = rng.uniform(0.2, 2.5, size=2)
        d, s, t = orc.dist_between_cells(r1, n1, h1, r2, n2, h2)
        d2, s2, t2 = orc.dist_between_cells(r2, n2, h2, r1, n1, h1)
        np.testing.assert_allclose(d, -d2, atol=1e-12)
        assert abs(s - t2) < 1e-10 and abs(t - s2) < 1e-10
        # brute force over a fine parameter grid never beats the closest points
        ss = np.linspace(-h1, h1, 201)[:, None, None]
        tt = np.linspace(-h2, h2, 201)[None, :, None]
        p = (r2 + tt * n2) - (r1 + ss * n1)
        assert np.sqrt((p ** 2).sum(-1)).min() >= np.linalg.norm(d) - 1e-12


def test_oracle_jkr_no_adhesion_limit():
    # testJKR.cpp:26-49: a = sqrt(R delta) at gamma = 0, tol 1e-8
    R, Rcell = 0.8, 0.5
    for delta in np.linspace(0, 2 * (R - Rcell), 100):
        a = orc.LIB.oracle_jkr_contact_radius(delta, R, 3900.0, 0.0)
        assert abs(a - math.sqrt(R * delta)) <= 1e-8


def test_oracle_jkr_adhesion_invariants():
    # testJKR.cpp:51-83: a >= sqrt(R delta) and delta = a^2/R - 2 sqrt(pi gamma a / E)
    R, Rcell, E0 = 0.8, 0.5, 3900.0
    for gamma in np.linspace(10, 100, 41):
        for delta in np.linspace(0, 2 * (R - Rcell), 100):
            a = orc.LIB.oracle_jkr_contact_radius(delta, R, E0, gamma)
            assert a >= math.sqrt(R * delta)
            rec = a * a / R - 2 * math.sqrt(math.pi * gamma * a / E0)
            assert abs(rec - delta) <= 1e-13 * max(1.0, a * a / R)


def _parteli_roots(delta, R, E, gamma):
    """Closed-form roots of a^4 - 2 R delta a^2 - (4 pi gamma R^2 / E) a + R^2 delta^2 = 0
    (Parteli et al. 2014), as testContactArea.cpp:138-150 writes them, in 60-digit mpmath."""
    import mpmath as mp
    with mp.workdps(60):
        d, R, E, g = mp.mpf(delta), mp.mpf(R), mp.mpf(E), mp.mpf(gamma)
        c0, c1, c2 = R * R * d * d, -4 * mp.pi * g * R * R / E, -2 * R * d
        P = -c2 * c2 / 12 - c0
        Q = -c2 ** 3 / 108 + c0 * c2 / 3 - c1 * c1 / 8
        U = mp.cbrt(-Q / 2 + mp.sqrt(Q * Q / 4 + P ** 3 / 27))
        s = -5 * c2 / 6 + (U - P / (3 * U))
        w = mp.sqrt(c2 + 2 * s)
        root = mp.sqrt(w * w - 4 * (c2 + s + c1 / (2 * w)))
        poly = lambda a: c0 + c1 * a + c2 * a * a + a ** 4
        return (w + root) / 2, (w - root) / 2, poly


def test_oracle_jkr_radius_matches_the_closed_form():
    # testContactArea.cpp:102-161 (jkrContactRadius): delta 0.1, R 0.8, E 3900, gamma 100; the
    # larger root exceeds the Hertz radius, zeroes the quartic and equals Parteli's a1 to 1e-15.
    # The table uses only the larger root (simulation.hpp:86-104), so the smaller one is not
    # compared.  The same bar over a grid of radii, adhesion energies and overlaps, for the
    # oracle and for the library's host solver (abm_jkr_contact_radius).
    import abm_b200
    import mpmath as mp
    a1, a2, poly = _parteli_roots(0.1, 0.8, 3900.0, 100.0)
    a = orc.LIB.oracle_jkr_contact_radius(0.1, 0.8, 3900.0, 100.0)
    assert a - math.sqrt(0.8 * 0.1) > 1e-15 and a2 > 1e-15
    with mp.workdps(60):
        assert abs(poly(mp.mpf(a))) < 1e-15
    assert abs(a - a1) < 1e-15
    for R in (0.4, 0.8):
        for gamma in (1.0, 10.0, 100.0, 1000.0):
            for delta in (1e-4, 0.01, 0.1, 0.3, 0.6):
                a1, _, _ = _parteli_roots(delta, R, 3900.0, gamma)
                assert abs(orc.LIB.oracle_jkr_contact_radius(delta, R, 3900.0, gamma) - a1) < 1e-15
                assert abs(abm_b200.jkr_contact_radius(delta, R, 3900.0, gamma) - a1) < 1e-15


def test_oracle_jkr_table_mesh():
    # simulation.hpp:1379-1382: LinSpaced(100, 0, 2 (R - Rcell)), last entry exactly 2 (R - Rcell)
    d, r = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)
    assert d[0] == 0.0 and d[-1] == 2 * (0.8 - 0.5)
    assert np.all(np.diff(d) > 0) and np.all(np.diff(r) > 0)


def _params(**kw):
    import abm_b200
    _, d = abm_b200.make_params(**kw)
    return d


def test_oracle_horizontal_cell_stationary():
    # testHorizontal.cpp:79-126: one non-growing horizontal cell just touching the
    # surface keeps x, y, orientation and length, and settles at
    # rz = R (1 - (sigma0 / (4 R E0))^(2/3))
    R, E0, sigma0, half_l = 0.8, 3900.0, 100.0, 0.5
    # (the reference test's 1e-7 step cap and 1e-10 tolerance pin dt at 1e-9 for the
    # whole run; a 1e-5 cap and 1e-8 tolerance reach the same equilibrium in 2000 steps)
    p = _params(adhesion_mode=0, max_stepsize=1e-5, min_stepsize=1e-9, max_error_allowed=1e-8,
                nz_threshold=1e-20, cell_surface_coulomb_coeff=0.0, L0=1.0, Ldiv=2 * (R + 1.0),
                neighbor_threshold=2 * (2 * R + 1.0))
    o = orc.Oracle(p)
    cells = np.zeros((1, 21))
    cells[0, [3, 4]] = [0.999 * R, 1.0]
    cells[0, 13], cells[0, 14] = 2 * half_l, half_l
    cells[0, 17], cells[0, 18], cells[0, 19], cells[0, 20] = 0.072, 720.0, sigma0, 1
    o.set_cells(cells)
    o.loop_init()
    o.iterate(2000)
    c = o.cells()
    tol = 1e-8
    assert abs(c[0, 1]) < tol and abs(c[0, 2]) < tol
    assert abs(c[0, 4] - 1) < tol and abs(c[0, 5]) < tol and abs(c[0, 6]) < tol
    assert abs(c[0, 13] - 2 * half_l) < tol and abs(c[0, 14] - half_l) < tol
    target = R * (1 - (0.25 * sigma0 / (R * E0)) ** (2.0 / 3.0))
    assert abs(c[0, 3] - target) < 1e-8


def test_oracle_velocity_identity():
    # testVelocities.cpp:40-131: M v = F + 2 lambda n for the full 3-D branch,
    # with M the composite viscosity matrix (mechanics.hpp:947-1009)
    R, eta0, eta1 = 0.8, 0.072, 720.0
    p = _params(adhesion_mode=0, cell_surface_coulomb_coeff=0.0)
    for j in range(10):
        ang = 0.5 * math.pi * (j + 1) / 10.0
        nz, half_l = math.sin(ang), 0.5
        rz = R + half_l * nz - 0.2 * R
        cells = np.zeros((1, 21))
        cells[0, 3:7] = [rz, math.cos(ang), 0.0, nz]
        cells[0, 13], cells[0, 14] = 2 * half_l, half_l
        cells[0, 17], cells[0, 18], cells[0, 19] = eta0, eta1, 100.0
        o = orc.Oracle(p)
        o.set_cells(cells)
        o.build_neighbors()
        v = o.get_velocities()[0]
        F = o.conservative_forces()[0]
        A = np.zeros(3)
        orc.LIB.oracle_area_integrals(rz, nz, R, half_l, A.ctypes.data_as(orc.ctypes.POINTER(orc.ctypes.c_double)))
        l = 2 * half_l
        t1, t2 = eta0 * l, eta0 * l ** 3 / 12
        t3, t4, t5 = (eta1 / R) * A
        M = np.zeros((6, 6))
        M[0, 0] = M[1, 1] = t1 + t3
        M[0, 3] = M[3, 0] = M[1, 4] = M[4, 1] = t4
        M[2, 2] = t1
        M[3, 3] = M[4, 4] = t2 + t5
        M[5, 5] = t2
        prod = M @ v
        n = cells[0, 4:7]
        np.testing.assert_allclose(prod[:3], F[:3], atol=1e-9 * max(1, abs(F).max()))
        lam = (prod[5] - F[5]) / (2 * nz)
        np.testing.assert_allclose(prod[3:5], F[3:5] + 2 * lam * n[:2], atol=1e-9 * max(1, abs(F).max()))


def test_deterministic_log_sincos_accuracy():
    # the division draws use series log / sin / cos evaluated identically on both sides;
    # they must still be accurate to a few ulp
    rng = np.random.default_rng(0)
    for u in np.concatenate([rng.random(2000), [2.2e-16, 1e-300, 0.5, 0.999999999999]]):
        assert abs(orc.LIB.oracle_det_log(u) - math.log(u)) <= 4e-16 * max(1.0, abs(math.log(u)))
    s, c = orc.ctypes.c_double(), orc.ctypes.c_double()
    for x in np.concatenate([rng.uniform(-7, 7, 2000), rng.uniform(0, 2 * math.pi, 500)]):
        orc.LIB.oracle_det_sincos(x, orc.ctypes.byref(s), orc.ctypes.byref(c))
        assert abs(s.value - math.sin(x)) <= 4e-16 and abs(c.value - math.cos(x)) <= 4e-16
