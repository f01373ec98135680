"""Cell-cell kinetic friction on the device (cellCellFrictionForces, mechanics.hpp:1031-1175,
added by cellCellInteractionForces when friction_mode is KINETIC, mechanics.hpp:1339-1346)
against the oracle's restatement, through the C ABI.  Bar: 1e-10 normwise (FP64), the
bar of the other FP64 parity tests.

Friction reads the stored velocities and the neighbor table, both fixed over an attempt;
the stage positions enter only through the planar-contact rule (|dz / d| < 1e-3 with both
contact points below 1.01 R, surface present), whose decision can change from stage to
stage.  The device computes both forces of every such candidate once per attempt and,
before the attempt, runs trial passes over the cells with candidates until every stage's
decision agrees with the stage states; the monolayer cases here put many contact points
within a stage's motion of the 1.01 R plane, so decisions do change between stages.
"""
import numpy as np
import pytest

import abm_b200
import oracle_ref as orc
from test_gpu_parity import colwise_relerr, patch_state

pytestmark = pytest.mark.gpu

R = 0.8
JKR = orc.jkr_table(R, 0.5, 3900.0, 100.0, 100)


def with_friction(cells, adhesion, seed):
    """Append the friction coefficient column (22 with adhesion, 21 without) and give the
    cells stored velocities (dn perpendicular to n)."""
    rng = np.random.default_rng(seed)
    n = len(cells)
    base = cells[:, :22] if adhesion else cells[:, :21]
    out = np.hstack([base, rng.uniform(1.0, 8.0, (n, 1))])
    out[:, 7:10] = rng.normal(0.0, 0.4, (n, 3))
    dn = rng.normal(0.0, 0.4, (n, 3))
    nn = out[:, 4:7]
    out[:, 10:13] = dn - (dn * nn).sum(1, keepdims=True) * nn
    return np.asfortranarray(out)


def monolayer(n_side=24, seed=7, spread=0.002):
    """Cells lying in the xy-plane on a lattice, touching end to end and side by side,
    with their contact points within `spread` of the 1.01 R plane."""
    rng = np.random.default_rng(seed)
    rows = []
    for a in range(n_side):
        for b in range(n_side):
            th = rng.uniform(-0.05, 0.05)
            z = 1.01 * R + rng.uniform(-spread, spread)
            rows.append(([a * 3.55, b * 1.52 + 0.3 * (a % 2), z], [np.cos(th), np.sin(th), 0.0]))
    cells = np.zeros((len(rows), 22))
    for k, (r, nv) in enumerate(rows):
        cells[k, 0] = k
        cells[k, 1:4] = r
        cells[k, 4:7] = nv
        cells[k, 13], cells[k, 14] = 2.0, 1.0
        cells[k, 17], cells[k, 18], cells[k, 19], cells[k, 20], cells[k, 21] = 100.0, 720.0, 100.0, 1, 100.0
    return cells


def pair(cells, **kw):
    kw.setdefault("cap_cells", len(cells) + 16)
    kw.setdefault("cell_cell_coulomb_coeff", 1.0)
    sim = abm_b200.Simulation(jkr_table=JKR, friction_mode=1, **kw)
    sim.upload_cells(cells)
    o = orc.Oracle(sim.pdict, jkr=JKR)
    o.set_cells(cells)
    return sim, o


def planar_decisions(cells, table):
    """Per neighbor row (i, j, d, s, t): the planar decision of the two contact points of
    `cells` (None where the contact is not a candidate)."""
    out = []
    for row in table:
        i, j = int(row[0]), int(row[1])
        d = row[2:5]
        if abs(d[2]) / np.linalg.norm(d) >= 1e-3 or np.linalg.norm(d) >= 2 * R:
            out.append(None)
            continue
        zi = cells[i, 3] + row[5] * cells[i, 6]
        zj = cells[j, 3] + row[6] * cells[j, 6]
        out.append(bool(zi < 1.01 * R and zj < 1.01 * R))
    return out


@pytest.mark.parametrize("adhesion", [0, 1])
@pytest.mark.parametrize("no_surface", [0, 1])
def test_friction_pair_forces_and_velocities(adhesion, no_surface):
    cells = with_friction(patch_state(2500, 71), adhesion, 71)
    sim, o = pair(cells, adhesion_mode=adhesion, no_surface=no_surface)
    assert sim.get_cell_neighbors() == o.build_neighbors()
    fo = o.cell_cell_forces()
    assert colwise_relerr(sim.cell_cell_forces(), fo) <= 1e-10
    # friction is in them: the forces without it differ
    plain = orc.Oracle(dict(sim.pdict, friction_mode=0), jkr=JKR)
    plain.set_cells(cells)
    plain.build_neighbors()
    assert colwise_relerr(plain.cell_cell_forces(), fo) > 1e-3
    assert colwise_relerr(sim.get_velocities(), o.get_velocities()) <= 1e-10
    sim.close()


@pytest.mark.parametrize("coeff", [0.0, 0.05])
def test_friction_coulomb_cap(coeff):
    cells = with_friction(patch_state(1500, 72), 1, 72)
    cells[:, 7:13] *= 50.0                            # fast sliding: the cap binds
    sim, o = pair(cells, adhesion_mode=1, cell_cell_coulomb_coeff=coeff)
    sim.get_cell_neighbors()
    o.build_neighbors()
    assert colwise_relerr(sim.cell_cell_forces(), o.cell_cell_forces()) <= 1e-10
    sim.close()


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
def test_friction_rk_attempt_with_planar_contacts(mode):
    """One RK attempt of a surface monolayer whose contact points straddle the 1.01 R plane,
    with vertical noise moving them by about the spread within a stage."""
    cells = with_friction(monolayer(), 0, 73)
    cells[:, 7:13] = 0.0
    cells[:, 7:9] = np.random.default_rng(3).normal(0.0, 0.5, (len(cells), 2))
    sim, o = pair(cells, adhesion_mode=0, integration_mode=mode, max_rz_noise=3000.0, rng_seed=11)
    assert sim.get_cell_neighbors() == o.build_neighbors()
    table = o.neighbors()
    d0 = planar_decisions(cells, table)
    assert sum(x is not None for x in d0) > 200            # many candidate contacts
    assert colwise_relerr(sim.cell_cell_forces(), o.cell_cell_forces()) <= 1e-10
    dt = 2e-4
    cg, eg, Eg = sim.step_runge_kutta_adaptive(dt)
    co, eo, Eo = o.rk_attempt(dt)
    assert colwise_relerr(cg, co) <= 1e-10
    # the embedded error estimates are differences of nearly equal stage sums (down to
    # 1e-20 here): held to FP64 rounding of the step, and E to the same in its units
    step = np.abs(co[:, 1:7] - cells[:, 1:7]).max()
    assert np.abs(eg - eo).max() <= 1e-10 * step
    assert abs(Eg - Eo) <= 1e-6 * max(abs(Eo), 1e-3)
    # the decisions at the end of the step differ from those at y0 for some contacts, so
    # the stages in between saw changed decisions too
    d1 = planar_decisions(co, table)
    changed = sum(1 for a, b in zip(d0, d1) if a is not None and a != b)
    print("\ncandidates %d, decisions changed over the step %d" % (sum(x is not None for x in d0), changed))
    assert changed > 0
    sim.close()


@pytest.mark.parametrize("graphs", [1, 0])
def test_friction_loop_matches_oracle(graphs):
    """Eight iterations of the loop (reference controller, dt adapting under 1e-4 h) on the
    monolayer: the same attempts, clock and state as the oracle's loop."""
    cells = with_friction(monolayer(16, 9), 0, 74)
    sim, o = pair(cells, adhesion_mode=0, integration_mode=2, max_rz_noise=2000.0, rng_seed=5,
                  max_stepsize=1e-4, iter_update_neighbors=4, use_graphs=graphs)
    sim.get_cell_neighbors()
    o.loop_init()
    for it in range(8):
        s = sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        assert colwise_relerr(cg, co) <= 1e-9, it
        assert np.array_equal(cg[:, 21], co[:, 21])      # the coefficient column travels
        t, dt, i = sim.clock()
        to, dto, io = o.clock()
        assert i == io and abs(dt - dto) <= 1e-9 * dto
    assert s["attempts"] == o.stats()["attempts"]
    sim.close()


def test_friction_with_division_keeps_coefficients():
    """Daughters inherit the mother's friction coefficient (growth.hpp:380-418 copies the
    mother's row)."""
    cells = with_friction(patch_state(300, 75), 1, 75)
    rng = np.random.default_rng(75)
    cells[:, 1:3] *= 2.0
    cells[:40, 13] = 5.65
    cells[:, 14] = cells[:, 13] / 2
    cells[:, 16] = 0.5
    sim, o = pair(cells, adhesion_mode=1, cap_cells=2 * len(cells), max_stepsize=1e-6, growth_mean=0.5)
    sim.set_parents(-np.ones(len(cells), dtype=np.int32))
    o.set_parents(-np.ones(len(cells), dtype=np.int32))
    sim.get_cell_neighbors()
    o.loop_init()
    sim.iterate(1)
    o.iterate(1)
    cg, co = sim.download_cells(), o.cells()
    assert len(cg) == len(co) == len(cells) + 40
    assert np.array_equal(cg[:, 22], co[:, 22])
    assert colwise_relerr(cg, co) <= 1e-9
    sim.close()


def test_friction_arguments_are_checked():
    with pytest.raises(RuntimeError):
        abm_b200.Simulation(jkr_table=JKR, friction_mode=1, precision=abm_b200.PRECISION_MIXED, cap_cells=16)
    with pytest.raises(RuntimeError):
        abm_b200.Simulation(jkr_table=JKR, friction_mode=2, cap_cells=16)
    sim = abm_b200.Simulation(jkr_table=JKR, friction_mode=1, cap_cells=16, adhesion_mode=1)
    with pytest.raises(RuntimeError, match="friction column"):
        sim.upload_cells(patch_state(10, 76)[:, :22])
    sim.close()


def test_friction_with_the_pi_controller():
    """Friction under a proposing controller (the PI rule): the trial passes run before the
    proposal's in-place attempt and before the retries that start from its backup."""
    cells = with_friction(monolayer(14, 11), 0, 77)
    sim, o = pair(cells, adhesion_mode=0, integration_mode=2, max_rz_noise=2000.0, rng_seed=6,
                  max_stepsize=1e-4, controller=abm_b200.CONTROLLER_PI)
    sim.get_cell_neighbors()
    o.loop_init()
    for it in range(8):
        sim.iterate(1)
        o.iterate(1)
        assert colwise_relerr(sim.download_cells(), o.cells()) <= 1e-9, it
    assert sim.stats()["attempts"] == o.stats()["attempts"]
    sim.close()


def test_friction_coefficients_travel_through_frames_and_compaction():
    """The coefficient column comes back in frames, and basal-only compaction keeps each
    kept cell's coefficient."""
    cells = with_friction(patch_state(800, 78), 1, 78)
    sim, o = pair(cells, adhesion_mode=1, max_stepsize=1e-5)
    sim.set_basal_only(True, 0.01)
    o.set_basal_only(True, 0.01)
    sim.set_frames(1e-5, slots=4)
    sim.get_cell_neighbors()
    o.loop_init()
    frames = 0
    for it in range(3):
        k0 = sim.frames_taken()
        sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        assert len(cg) == len(co)
        assert np.array_equal(cg[:, 0], co[:, 0]) and np.array_equal(cg[:, 22], co[:, 22])
        assert colwise_relerr(cg, co) <= 1e-9
        if sim.frames_taken() > k0:                 # a frame of this iteration's end state
            fc = sim.download_frame(sim.frames_taken() - 1)[0]
            assert np.array_equal(fc[:, 22], cg[:, 22])
            frames += 1
    assert len(cg) < len(cells) and frames >= 1
    sim.close()
