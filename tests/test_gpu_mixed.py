"""Parity of the mixed-precision path (ABM_PRECISION_MIXED, the benchmark's chosen
arm) with the FP64 CPU oracle, through the C ABI.

What runs in FP32 there: the closest-point solve of skew segment pairs with
|cos| < 0.99, the Hertz force law, and the surface forces and velocity solve of cells
in surface contact.  What stays FP64: the neighbor decisions (exact FP64 distance),
the distance vector and overlap, the JKR magnitude, the near-parallel pairs,
positions, orientations, stage sums and the error norm.

Bars, stated here:
  * neighbor pair set and the table's (d, s, t): bit for bit, as in FP64;
  * pair forces dE/dq and velocities: normwise relative error per column
    max|mixed - oracle| / max|oracle| <= 1e-4 (measured: 3e-6 and 8e-6 on the 100k state);
  * one RK step, in the error test's own units (simulation.hpp:1697-1705):
    max_i |y1_mixed - y1_oracle| / (tol (1 + |y0|)) <= 0.05, i.e. the FP32 rounding
    moves the step by at most 5 % of what the error test accepts (measured: 0.011 at
    dt = 1e-6 h on the 100k state, 0.02 at 1e-5 h on a 3000-cell patch); and the scaled error
    norm E agrees to 1e-3 relative above a floor of 1e-3: the FP32 stage velocities of
    cells in surface contact put rounding noise into the embedded error, about
    eps_32 |k| dt / (tol (1 + |y|)) (measured up to 1.8e-4 at dt = 1e-5 h, where the FP64
    oracle's E is 6e-12), which matters only where E itself is that small (high-order
    tableaux at small dt), three orders below the accept threshold E = 1.
"""
import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc
from test_gpu_parity import colwise_relerr, parallel_bundle, patch_state

pytestmark = pytest.mark.gpu

JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)
TOL = 1e-8
RTOL_FORCE = 1e-4
RK_UNITS_MAX = 0.05
E_RTOL = 1e-3
E_FLOOR = 1e-3


def rk_units(c_mixed, c_oracle, cells, tol=TOL):
    """max over cells and the six coordinates of |y1_mixed - y1_oracle| / (tol (1 + |y0|))."""
    y0 = cells[:, 1:7]
    return float((np.abs(c_mixed[:, 1:7] - c_oracle[:, 1:7]) / (tol * (1 + np.abs(y0)))).max())


def mixed_and_oracle(cells, **kw):
    kw.setdefault("cap_cells", max(len(cells), 1) + 16)
    sim = abm_b200.Simulation(jkr_table=JKR, precision=abm_b200.PRECISION_MIXED, max_error_allowed=TOL, **kw)
    sim.upload_cells(cells)
    o = orc.Oracle(sim.pdict, jkr=JKR)
    o.set_cells(cells)
    return sim, o


def check_state(cells, dts=(1e-6,), **kw):
    sim, o = mixed_and_oracle(cells, **kw)
    m = sim.get_cell_neighbors()
    assert m == o.build_neighbors() and m > 0
    assert np.array_equal(sim.neighbors(), o.neighbors())       # decisions stay FP64
    ef = colwise_relerr(sim.cell_cell_forces(), o.cell_cell_forces())
    ev = colwise_relerr(sim.get_velocities(), o.get_velocities())
    assert ef <= RTOL_FORCE, ef
    assert ev <= RTOL_FORCE, ev
    out = []
    for dt in dts:
        cg, _, Eg = sim.step_runge_kutta_adaptive(dt)
        co, _, Eo = o.rk_attempt(dt)
        u = rk_units(cg, co, cells)
        print("\nmixed vs oracle at dt %g: forces %.2e, velocities %.2e, step %.3e of tol, E %.6g vs %.6g"
              % (dt, ef, ev, u, Eg, Eo))
        assert u <= RK_UNITS_MAX, u
        assert abs(Eg - Eo) <= E_RTOL * Eo + E_FLOOR, (Eg, Eo)
        # the columns the step does not move are copied unchanged
        assert np.array_equal(cg[:, 13:], co[:, 13:])
        out.append((u, Eg, Eo))
    sim.close()
    return out


def test_mixed_full_size_state():
    """The benchmark's own 100k-cell state (centres in a 300 um disk, z in [R, 10])."""
    cells, _ = workloads.biofilm_3d(n=100000, seed=1, p_contact=0.9)
    check_state(cells, dts=(1e-6,))


@pytest.mark.parametrize("jitter", [0.0, 0.004])
def test_mixed_near_parallel_bundle(jitter):
    """Cells along x on a lattice: the near-parallel branch (|n1 . n2| >= 0.9999) stays FP64."""
    check_state(parallel_bundle(jitter=jitter), dts=(1e-6, 1e-5))


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
def test_mixed_rk_attempt_all_tableaux(mode):
    check_state(patch_state(3000, 13), dts=(1e-6, 1e-5), integration_mode=mode)


def test_mixed_loop_matches_oracle_loop():
    """Twenty iterations of the loop body (reference controller, mixed precision) from one
    state with dt held at 1e-6 h as in the benchmark: the same attempts as the FP64
    oracle, and the cells within twenty steps' worth of the per-step bound."""
    cells = patch_state(2000, 21)
    sim, o = mixed_and_oracle(cells, iter_update_neighbors=10, max_stepsize=1e-6)
    sim.get_cell_neighbors()
    o.loop_init()
    s = sim.iterate(20)
    o.iterate(20)
    assert s["attempts"] == o.stats()["attempts"]
    t, dt, it = sim.clock()
    to, dto, ito = o.clock()
    assert it == ito and dt == dto and abs(t - to) <= 1e-12 * to
    cg, co = sim.download_cells(), o.cells()
    assert rk_units(cg, co, cells) <= 20 * RK_UNITS_MAX
    assert np.array_equal(sim.neighbors()[:, :2], o.neighbors()[:, :2])
    sim.close()


def test_mixed_loop_takes_the_oracle_decisions():
    """With dt free to adapt (cap 1e-4 h) the mixed path accepts and rejects the same
    attempts as the FP64 oracle over twenty iterations; its step sizes, set from E, stay
    within 1 % of the oracle's."""
    cells = patch_state(2000, 22)
    sim, o = mixed_and_oracle(cells, iter_update_neighbors=10, max_stepsize=1e-4)
    sim.get_cell_neighbors()
    o.loop_init()
    s = sim.iterate(20)
    o.iterate(20)
    assert s["attempts"] == o.stats()["attempts"]
    t, dt, it = sim.clock()
    to, dto, ito = o.clock()
    assert it == ito and abs(dt - dto) <= 1e-2 * dto and abs(t - to) <= 1e-2 * to
    sim.close()
