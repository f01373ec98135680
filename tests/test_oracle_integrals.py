"""The oracle's surface integrals (integrals.hpp, restated in oracle/abm3d.hpp) pinned
the way the reference's own tests pin them (ABM-3d/ABM-3d-cpp/test/src/testIntegrals.cpp):
each closed form against a quadrature of its integrand along the cell, for the
exponents 0.5, 1, 1.5, 2 and ten orientations nz = sin(pi/2 (i + 1) / 10), with a cell
overlapping the surface by at most 0.2 R and with a cell 0.1 R clear of it (zero), at
the tolerances asserted there (1e-8 for integral1/2, 1e-7 for the others).  The
reference integrates with a trapezoid rule of up to 1e9 points in 100-digit MPFR;
adaptive quadrature with a breakpoint where the overlap reaches zero stands in here."""
import math

import pytest
from scipy import integrate

import oracle_ref as orc

R = 0.8
HALF_L = 0.5
EXPONENTS = (0.5, 1.0, 1.5, 2.0)
NZ = [math.sin(math.pi / 2 * (i + 1) / 10) for i in range(10)]
CASES = {"contact": 0.2 * R, "clear": -0.1 * R}       # maximum overlap of the cell


def geometry(nz, max_overlap):
    rz = R + HALF_L * nz - max_overlap                   # testIntegrals.cpp:116-118, :132-134
    return rz, (R - rz) / nz


def quad(f, rz, nz):
    ss = (R - rz) / nz                                   # where the overlap R - rz - s nz reaches 0
    pts = [ss] if -HALF_L < ss < HALF_L else None
    val, _ = integrate.quad(f, -HALF_L, HALF_L, points=pts, epsabs=1e-13, epsrel=1e-13, limit=200)
    return val


def overlap(rz, nz, s):
    return R - rz - s * nz


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("gamma", EXPONENTS)
def test_integral1_and_2(case, gamma):
    for nz in NZ:
        rz, ss = geometry(nz, CASES[case])
        f1 = lambda s: max(overlap(rz, nz, s), 0.0) ** gamma
        f2 = lambda s: s * max(overlap(rz, nz, s), 0.0) ** gamma
        t1, t2 = quad(f1, rz, nz), quad(f2, rz, nz)
        assert abs(orc.LIB.oracle_integral1(rz, nz, R, HALF_L, gamma, ss) - t1) < 1e-8
        assert abs(orc.LIB.oracle_integral2(rz, nz, R, HALF_L, gamma, ss) - t2) < 1e-8
        if case == "clear":
            assert t1 == 0.0 and t2 == 0.0


@pytest.mark.parametrize("case", sorted(CASES))
def test_integrals_4_5_6(case):
    for nz in NZ:
        rz, ss = geometry(nz, CASES[case])
        step = lambda s: 1.0 if overlap(rz, nz, s) > 0 else 0.0
        for k, g in ((4, lambda s: step(s)), (5, lambda s: s * step(s)), (6, lambda s: s * s * step(s))):
            got = getattr(orc.LIB, "oracle_integral%d" % k)(nz, HALF_L, ss)
            assert abs(got - quad(g, rz, nz)) < 1e-7, (k, nz)


@pytest.mark.parametrize("case", sorted(CASES))
def test_area_integrals(case):
    import numpy as np
    for nz in NZ:
        rz, ss = geometry(nz, CASES[case])

        def a(s):
            d = overlap(rz, nz, s)
            return (math.sqrt(R) * (1 - nz * nz) * math.sqrt(max(d, 0.0))
                    + math.pi * R * nz * nz * (1.0 if d > 0 else 0.0))
        out = np.zeros(3)
        orc.LIB.oracle_area_integrals(rz, nz, R, HALF_L, orc._dp(out))
        for k, w in enumerate((lambda s: 1.0, lambda s: s, lambda s: s * s)):
            target = quad(lambda s: w(s) * a(s), rz, nz)
            assert abs(out[k] - target) < 1e-7, (k, nz)
