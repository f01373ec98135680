"""The adhesion energy density for a target equilibrium distance: the library's closed form
(abm_jkr_optimal_gamma) against the oracle's restatement of the reference's nested Newton
solves (jkrOptimalSurfaceEnergyDensity / jkrEquilibriumDistance, jkr.hpp:1311-1407, with the
arguments of simulation.hpp:1355-1358).  Host code only.

  * At every target the reference's procedure solves, the oracle's gamma puts the equilibrium
    within the reference's stopping tolerance (1e-8) of the target, and the two gammas differ by
    no more than that tolerance allows (d gamma / gamma = 1.5 d(delta) / delta).
  * The library's gamma balances the JKR force exactly: the oracle's equilibrium distance at it
    is the target to 1e-11, and the force at the target overlap is zero to rounding.
  * At the overlap cap 2 (R - Rcell) every larger gamma gives the same capped distance; the
    library returns the smallest, the edge of that plateau.
  * Targets just above 2 Rcell, from which the reference's first Newton step lands on the
    capped plateau and its finite-difference derivative is zero (eqdist below ~1.19 for
    R = 0.8, Rcell = 0.5, E0 = 3900), have no reference result to compare; the library's
    force balance is checked there alone."""
import math

import numpy as np
import pytest

import abm_b200
import oracle_ref as orc

R, RCELL, E0 = 0.8, 0.5, 3900.0


def balance(gamma, eqdist):
    a = orc.LIB.oracle_jkr_contact_radius(2 * R - eqdist, R / 2, E0, gamma)
    hertz = (4.0 / 3.0) * E0 / (R / 2) * a ** 3
    return hertz - 4 * math.sqrt(math.pi * gamma * E0) * a ** 1.5, hertz


@pytest.mark.parametrize("eqdist", [1.2, 1.3, 1.4, 1.5, 1.55, 1.58, 1.59, 1.599])
def test_closed_form_matches_the_reference_procedure(eqdist):
    g_lib = abm_b200.jkr_optimal_gamma(R, RCELL, E0, eqdist)
    g_ref = orc.LIB.oracle_jkr_optimal_gamma(R, RCELL, E0, eqdist)
    assert abs(orc.LIB.oracle_jkr_equilibrium_distance(R, RCELL, E0, g_ref) - eqdist) <= 1e-8
    assert abs(orc.LIB.oracle_jkr_equilibrium_distance(R, RCELL, E0, g_lib) - eqdist) <= 1e-11
    delta = 2 * R - eqdist
    assert abs(g_lib - g_ref) <= 1.5 * 1.01 * 1e-8 / delta * g_lib, (g_lib, g_ref)


@pytest.mark.parametrize("eqdist", [1.0 + 1e-9, 1.01, 1.05, 1.1, 1.15, 1.2, 1.45, 1.6 - 1e-6])
def test_closed_form_balances_the_jkr_force(eqdist):
    g = abm_b200.jkr_optimal_gamma(R, RCELL, E0, eqdist)
    force, hertz = balance(g, eqdist)
    assert abs(force) <= 1e-12 * hertz
    # the reference's inner solve stops at |force| <= 1e-8; below an overlap of ~1e-4 the force
    # is so flat that this leaves more than 1e-11 of slack in the distance it returns
    if 2 * R - eqdist >= 1e-4:
        assert abs(orc.LIB.oracle_jkr_equilibrium_distance(R, RCELL, E0, g) - eqdist) <= 1e-11


def test_overlap_cap_and_out_of_range_targets():
    cap_target = 2 * RCELL
    g = abm_b200.jkr_optimal_gamma(R, RCELL, E0, cap_target)
    assert abs(orc.LIB.oracle_jkr_equilibrium_distance(R, RCELL, E0, g) - cap_target) <= 1e-12
    assert orc.LIB.oracle_jkr_equilibrium_distance(R, RCELL, E0, 0.999 * g) > cap_target + 1e-4
    # on the plateau: the reference's answer is some gamma at or above the edge
    assert orc.LIB.oracle_jkr_optimal_gamma(R, RCELL, E0, cap_target) >= g
    for bad in (2 * R, 2 * R + 0.1, 2 * RCELL - 1e-3, 0.0):
        with pytest.raises(RuntimeError, match="ABM_ERR_ARG"):
            abm_b200.jkr_optimal_gamma(R, RCELL, E0, bad)


def test_set_gamma_from_eqdist_follows_the_driver():
    """simulation.hpp:1366-1371: group-1 cells get max_gamma, every other group 0."""
    cells = np.zeros((5, 22))
    cells[:, 20] = [1, 2, 1, 3, 2]
    cells[:, 21] = 7.0
    g = abm_b200.set_gamma_from_eqdist(cells, R, RCELL, E0, 1.5)
    assert g == abm_b200.jkr_optimal_gamma(R, RCELL, E0, 1.5)
    assert list(cells[:, 21]) == [g, 0.0, g, 0.0, 0.0]
