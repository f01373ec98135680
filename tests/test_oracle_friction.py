"""The oracle's cell-cell kinetic friction (cellCellFrictionForces, mechanics.hpp:1031-1175, added
by cellCellInteractionForces when friction_mode is KINETIC, mechanics.hpp:1339-1346).  The
reference has no test of this function, so its restatement is held to closed forms and to the
properties the model has by construction:

  * two overlapping cells sliding past each other: the force on each is
    -eta sqrt(Req overlap) times its tangential relative velocity, eta the smaller coefficient;
  * the Coulomb cap: at high sliding speed the force norm is coeff (4/3) E0 sqrt(Req) overlap^(3/2);
  * near the surface a nearly horizontal contact is taken in the xy-plane: no z force, the
    in-plane distance for the overlap; with the surface off the same contact keeps its z part;
  * on a random colony: forces cancel in pairs (Newton's third law), and the power the
    friction exerts on the cells' own velocities is never positive;
  * getConservativeForces subtracts it with the other pair forces, at every RK stage, so a run
    with friction differs from one without and repeats bit for bit.
This is the oracle side of the friction row; parity of a device kernel is not claimed here."""
import math

import numpy as np
import pytest

import oracle_ref as orc
from abm_b200 import workloads

R, E0 = 0.8, 3900.0
REQ = R / 2


def params(**kw):
    import abm_b200
    args = dict(adhesion_mode=0, nz_threshold=1e-8, no_surface=1)
    args.update({k: v for k, v in kw.items() if k not in ("friction_mode", "cell_cell_coulomb_coeff")})
    _, p = abm_b200.make_params(**args)
    p["friction_mode"] = kw.get("friction_mode", 1)
    p["cell_cell_coulomb_coeff"] = kw.get("cell_cell_coulomb_coeff", 0.0)
    return p


def pair_cells(r2, n2, v2, eta=(5.0, 3.0), z=1.1 * R, half_l=0.5):
    """Cell 0 at (0, 0, z) along x at rest, cell 1 at r2 along n2 moving with dr = v2;
    22 columns, the friction coefficient in column 21 (adhesion off)."""
    c = np.zeros((2, 22))
    c[0, 1:7] = [0, 0, z, 1, 0, 0]
    c[1, 0] = 1
    c[1, 1:4], c[1, 4:7], c[1, 7:10] = r2, n2, v2
    c[:, 13], c[:, 14] = 2 * half_l, half_l
    c[:, 17], c[:, 18], c[:, 19], c[:, 20] = 0.072, 720.0, 100.0, 1
    c[:, 21] = eta
    return c


def friction_part(p, cells):
    """dE/dq of the friction alone: the pair forces with it minus the pair forces without."""
    out = []
    for mode in (1, 0):
        q = dict(p, friction_mode=mode)
        o = orc.Oracle(q)
        o.set_cells(cells)
        o.build_neighbors()
        out.append(o.cell_cell_forces())
    return out[0] - out[1], o


def test_sliding_pair_closed_form():
    d, u = 1.4, 0.37
    cells = pair_cells((0.0, d, 1.1 * R), (1.0, 0.0, 0.0), (u, 0.0, 0.0))
    fr, o = friction_part(params(), cells)
    row = o.neighbors()[0]
    assert row[0] == 1 and row[1] == 0                  # i = 1 (moving), j = 0
    si, sj = row[5], row[6]
    mag = 3.0 * math.sqrt(REQ * (2 * R - d)) * u        # eta = min(5, 3)
    # force on cell 1 is -mag x (it is held back), on cell 0 +mag x; dE/dq is minus that
    expect = np.zeros((2, 6))
    expect[1, 0], expect[1, 3] = mag, si * mag
    expect[0, 0], expect[0, 3] = -mag, sj * mag
    np.testing.assert_allclose(fr, expect, rtol=1e-12, atol=1e-12 * mag)


def test_coulomb_cap():
    d, u, coeff = 1.4, 1e6, 0.5
    cells = pair_cells((0.0, d, 1.1 * R), (1.0, 0.0, 0.0), (u, 0.0, 0.0))
    fr, _ = friction_part(params(cell_cell_coulomb_coeff=coeff), cells)
    cap = coeff * (4.0 / 3.0) * E0 * math.sqrt(REQ) * (2 * R - d) ** 1.5
    assert abs(np.linalg.norm(fr[1, :3]) - cap) <= 1e-12 * cap
    fr_free, _ = friction_part(params(cell_cell_coulomb_coeff=0.0), cells)
    assert np.linalg.norm(fr_free[1, :3]) > 1e3 * cap  # uncapped without the coefficient


@pytest.mark.parametrize("no_surface", [0, 1])
def test_contact_near_the_surface_is_planar(no_surface):
    z, d, tilt = 0.95 * R, 1.4, 5e-4                    # contact points below 1.01 R, |dz/d| < 1e-3
    v2 = (0.2, 0.0, 0.3)
    cells = pair_cells((0.0, d, z + tilt * d), (1.0, 0.0, 0.0), v2, z=z)
    fr, o = friction_part(params(no_surface=no_surface), cells)
    row = o.neighbors()[0]
    dvec = row[2:5]
    assert abs(dvec[2]) / np.linalg.norm(dvec) < 1e-3
    if no_surface:
        assert abs(fr[1, 2]) > 1e-3 * abs(fr[1, 0])     # the z sliding is resisted too
    else:
        assert fr[1, 2] == 0 and fr[0, 2] == 0
        overlap = 2 * R - math.hypot(dvec[0], dvec[1])
        mag = 3.0 * math.sqrt(REQ * overlap) * v2[0]
        assert abs(fr[1, 0] - mag) <= 1e-12 * mag


@pytest.mark.parametrize("coeff", [0.0, 0.3])
def test_pairwise_cancellation_and_dissipation(coeff):
    cells, _ = workloads.biofilm_3d(n=400, seed=11, disk_radius=40 * math.sqrt(400 / 1e5) * 10, p_contact=0.9)
    rng = np.random.default_rng(3)
    cells = np.hstack([cells[:, :21], rng.uniform(1.0, 10.0, (len(cells), 1))])
    cells[:, 7:10] = rng.normal(0, 0.5, (len(cells), 3))
    dn = rng.normal(0, 0.5, (len(cells), 3))
    n = cells[:, 4:7]
    cells[:, 10:13] = dn - (dn * n).sum(1, keepdims=True) * n       # dn perpendicular to n
    fr, o = friction_part(params(cell_cell_coulomb_coeff=coeff), cells)
    assert np.count_nonzero(np.abs(fr).sum(1)) > 50
    scale = np.abs(fr[:, :3]).sum()
    assert np.all(np.abs(fr[:, :3].sum(0)) <= 1e-12 * scale)         # Newton's third law
    power = -(fr[:, :3] * cells[:, 7:10]).sum() - (fr[:, 3:] * cells[:, 10:13]).sum()
    assert power < 0 and power <= 1e-12 * np.abs(fr).sum()


def test_enters_conservative_forces_and_the_loop():
    cells = pair_cells((0.0, 1.4, 1.1 * R), (1.0, 0.0, 0.0), (0.3, 0.0, 0.1))
    base = params(max_stepsize=1e-6, max_error_allowed=1e-8)
    o_on, o_off = orc.Oracle(dict(base, friction_mode=1)), orc.Oracle(dict(base, friction_mode=0))
    for o in (o_on, o_off):
        o.set_cells(cells)
        o.build_neighbors()
    fr = o_on.cell_cell_forces() - o_off.cell_cell_forces()
    np.testing.assert_allclose(o_on.conservative_forces() - o_off.conservative_forces(), -fr,
                               rtol=1e-12, atol=1e-12 * np.abs(fr).max())
    ends = []
    for mode in (1, 1, 0):
        o = orc.Oracle(dict(base, friction_mode=mode))
        o.set_cells(cells)
        o.loop_init()
        o.iterate(50)
        ends.append(o.cells())
    assert np.array_equal(ends[0], ends[1])
    assert np.all(np.isfinite(ends[0])) and not np.array_equal(ends[0], ends[2])


def test_missing_friction_column_is_an_error_not_a_crash():
    cells = pair_cells((0.0, 1.4, 1.1 * R), (1.0, 0.0, 0.0), (0.3, 0.0, 0.0))[:, :21]
    o = orc.Oracle(params())
    o.set_cells(cells)
    o.build_neighbors()
    for call in (o.cell_cell_forces, o.conservative_forces, o.get_velocities):
        with pytest.raises(RuntimeError, match="friction column"):
            call()
