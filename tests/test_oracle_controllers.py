"""The oracle's step-size controllers on the CPU: the reference rule of
simulation.hpp:1688-1769 (trial + unconditional final re-run) and the PI controller
(a proposal accepted as is when its scaled error passes, the next dt from
dt 0.9 E_n^(-0.7/k) E_(n-1)^(0.4/k) within [0.2, 10] x dt and [min, max] step size)."""
import math

import numpy as np

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0)


def colony(n=300, seed=4):
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=300 * math.sqrt(n / 1e5), p_contact=0.9)
    return cells


def pi_next(dt, E, E_prev, k, lo, hi):
    f = 0.9 * (1.0 / E) ** (0.7 / k) * (E_prev if E_prev > 0 else 1.0) ** (0.4 / k)
    f = min(max(f, 0.2), 10.0)
    return min(max(dt * f, lo), hi)


def test_pi_proposal_follows_the_formula():
    cells = colony()
    _, p = abm_b200.make_params(controller=abm_b200.CONTROLLER_PI, max_stepsize=1e-3, min_stepsize=1e-9)
    o = orc.Oracle(p, jkr=JKR)
    o.set_cells(cells)
    o.loop_init()
    o.set_clock(0.0, 1e-7, 0)
    E_prev, dt = 0.0, 1e-7
    attempts = checked = 0
    for it in range(12):
        o.iterate(1)
        s = o.stats()
        E = s["last_max_error"]
        used = s["attempts"] - attempts
        attempts = s["attempts"]
        _, dt_now, _ = o.clock()
        if used == 1:
            # the proposal passed: accepted as is, then the PI step from it
            assert E <= 1.0
            expect = pi_next(dt, E, E_prev, 2, 1e-9, 1e-3)
            assert abs(dt_now - expect) <= 1e-14 * expect
            checked += 1
        E_prev, dt = E, dt_now
    assert checked >= 8 and dt > 1e-6          # dt grew by the PI factor from 1e-7 h


def test_pi_takes_one_attempt_per_passing_step_and_the_reference_two():
    cells = colony()
    out = {}
    for ctl in (abm_b200.CONTROLLER_REFERENCE, abm_b200.CONTROLLER_PI):
        _, p = abm_b200.make_params(controller=ctl, max_stepsize=1e-6)
        o = orc.Oracle(p, jkr=JKR)
        o.set_cells(cells)
        o.loop_init()
        o.iterate(10)
        out[ctl] = o.stats()
        t, dt, it = o.clock()
        assert it == 10 and dt == 1e-6          # the cap binds: E is far below 1 at 1e-6 h
    assert out[abm_b200.CONTROLLER_REFERENCE]["attempts"] == 20
    assert out[abm_b200.CONTROLLER_PI]["attempts"] == 10
    assert out[abm_b200.CONTROLLER_PI]["rejected"] == 0


def test_pi_rejection_continues_with_the_reference_rule():
    # a proposal far too large fails; the reference rule then retries and re-runs
    cells = colony()
    _, p = abm_b200.make_params(controller=abm_b200.CONTROLLER_PI, max_stepsize=1.0)
    o = orc.Oracle(p, jkr=JKR)
    o.set_cells(cells)
    o.loop_init()
    o.set_clock(0.0, 1e-2, 0)
    o.iterate(1)
    s = o.stats()
    assert s["rejected"] == 1 and s["attempts"] >= 3
    _, dt, _ = o.clock()
    assert dt < 1e-2
    assert np.isfinite(o.cells()).all()
