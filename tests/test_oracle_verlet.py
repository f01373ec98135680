"""The oracle's velocity-Verlet step (stepVelocityVerlet, mechanics.hpp:2668-2996, the
integration mode 0 branch of runSimulation, simulation.hpp:1279-1290 and 1786-1798) and the
include_constraint forms of the forces it uses.  The reference has no test of this integrator,
so the restatement is held to what the scheme guarantees:

  * with every dissipative term off (no surface, no ambient viscosity, no adhesion), a collision
    of two cells that sets both translating and turning conserves kinetic (translational and
    rotational, with the reference's moments of inertia) plus Hertz energy
    (8/15) E0 sqrt(Req) overlap^(5/2), to second order in dt, and total momentum exactly;
  * a lone cell drifting through the ambient fluid slows as exp(-eta0 l^3 t / m): the reference
    scales the ambient drag by the cube of the length (ambientViscosityForces computes
    li = pow(l, 3) and uses eta0 li dr), and the restatement keeps that;
  * the constrained cell-surface repulsion torque is the torque of the repulsive force density
    about the cell center, n x z times the integral of s f(s) (mechanics.hpp:741-755);
  * the driver's requirement that a cell mass be given (simulation.hpp:1283-1286).
This is the oracle side of the velocity-Verlet row; no device kernel is claimed."""
import ctypes
import math

import numpy as np
import pytest
from scipy import integrate

import oracle_ref as orc

R, RCELL, E0, HALF_L = 0.8, 0.5, 3900.0, 0.5


def params(dt, M0=1.0, L0=1.0, **kw):
    import abm_b200
    args = dict(adhesion_mode=0, no_surface=1, max_stepsize=dt, L0=L0, Ldiv=100.0,
                neighbor_threshold=2 * (2 * R + 2.0), iter_update_neighbors=10 ** 9, growth_mean=0.0,
                growth_std=0.0, Rcell=RCELL, E0=E0)
    args.update(kw)
    _, p = abm_b200.make_params(**args)
    p["integration_mode"], p["M0"] = 0, M0
    return p


def moment_perp(M0, L0, length):
    rho = M0 / (math.pi * (4.0 / 3.0 * R ** 3 + R * R * L0))
    d = 2 * R
    return rho * math.pi * d * d * (4 * d ** 3 + 15 * length * d * d + 20 * length ** 2 * d + 10 * length ** 3) / 480


def collision(dt, t_end=0.4):
    """Cell 0 along x, cell 1 along y in an offset T overlapping it by 0.1, both at rest."""
    cells = np.zeros((2, 21))
    cells[0, 1:7] = [0, 0, 5, 1, 0, 0]
    cells[1, 0] = 1
    cells[1, 1:7] = [HALF_L + 1.5, 0.25, 5, 0, 1, 0]
    cells[:, 13], cells[:, 14] = 2 * HALF_L, HALF_L
    o = orc.Oracle(params(dt))
    o.set_cells(cells)
    o.loop_init()
    inertia = moment_perp(1.0, 1.0, 2 * HALF_L)

    def energy(c):
        v, _, _ = orc.dist_between_cells(c[0, 1:4], c[0, 4:7], HALF_L, c[1, 1:4], c[1, 4:7], HALF_L)
        overlap = max(2 * R - np.linalg.norm(v), 0.0)
        e = (8.0 / 15.0) * E0 * math.sqrt(R / 2) * overlap ** 2.5
        for i in range(2):
            w = np.cross(c[i, 4:7], c[i, 10:13])
            e += 0.5 * np.dot(c[i, 7:10], c[i, 7:10]) + 0.5 * inertia * np.dot(w, w)
        return e

    series = [energy(o.cells())]
    for _ in range(int(round(t_end / dt))):
        o.iterate(1)
        series.append(energy(o.cells()))
    return np.array(series), o.cells()


def test_collision_conserves_energy_to_second_order():
    errs = []
    for dt in (4e-4, 2e-4, 1e-4):
        e, end = collision(dt)
        errs.append(np.abs(e - e[0]).max() / e[0])
    assert errs[-1] < 1e-5
    assert 3.5 < errs[0] / errs[1] < 4.5 and 3.5 < errs[1] / errs[2] < 4.5, errs
    assert np.all(np.abs(end[:, 7:10].sum(0)) <= 1e-12)            # momentum
    omega = np.cross(end[1, 4:7], end[1, 10:13])
    assert np.linalg.norm(omega) > 0.5                              # the collision set cell 1 turning
    assert np.allclose(np.linalg.norm(end[:, 4:7], axis=1), 1.0, atol=1e-14)


def test_ambient_drag_scales_with_the_cube_of_the_length():
    length, eta0, v0, dt, t_end = 2.0, 0.1, 0.5, 1e-3, 1.0
    cells = np.zeros((1, 21))
    cells[0, 1:7] = [0, 0, 5, 1, 0, 0]
    cells[0, 7] = v0
    cells[0, 13], cells[0, 14], cells[0, 17] = length, length / 2, eta0
    o = orc.Oracle(params(dt, M0=1.0, L0=length))                 # mass 1 at this length
    o.set_cells(cells)
    o.loop_init()
    o.iterate(int(round(t_end / dt)))
    v = o.cells()[0, 7]
    expect = v0 * math.exp(-eta0 * length ** 3 * t_end)
    assert abs(v - expect) < 1e-3 * expect, (v, expect)
    assert abs(v - v0 * math.exp(-eta0 * length * t_end)) > 0.1 * v0  # not the length-linear drag


@pytest.mark.parametrize("angle_i", [2, 5, 8])
def test_constrained_surface_repulsion_torque_is_the_moment_of_the_force_density(angle_i):
    angle = math.pi / 2 * (angle_i + 1) / 10
    nx, nz = math.cos(angle), math.sin(angle)
    rz = R + HALF_L * nz - 0.2 * R
    depth = lambda s: max(R - rz - s * nz, 0.0)
    density = lambda s: 2 * E0 * ((1 - nz * nz) * depth(s) + math.sqrt(R) * nz * nz * math.sqrt(depth(s)))
    ss = (R - rz) / nz
    pts = [ss] if -HALF_L < ss < HALF_L else None
    fz = integrate.quad(density, -HALF_L, HALF_L, points=pts, epsabs=1e-12, epsrel=1e-12)[0]
    moment = integrate.quad(lambda s: s * density(s), -HALF_L, HALF_L, points=pts, epsabs=1e-12, epsrel=1e-12)[0]
    out = {}
    for constraint in (0, 1):
        rep = np.zeros(6)
        orc.LIB.oracle_surface_forces(0, rz, nx, nz, HALF_L, 0.0, R, E0, 1e-8, constraint,
                                      rep.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        out[constraint] = rep
    # the z force is the integral of the density in both forms
    assert abs(-out[0][2] - fz) <= 1e-9 * fz and out[1][2] == out[0][2]
    # constrained: torque (n x z) * moment = (ny, -nx, 0) * moment, nothing about z
    np.testing.assert_allclose(-out[1][3:6], [0.0, -nx * moment, 0.0], rtol=1e-9, atol=1e-9 * abs(moment))
    assert out[0][3] == 0 and out[0][4] == 0 and out[0][5] != 0   # unconstrained: the nz row instead


def test_velocity_verlet_needs_a_cell_mass():
    cells = np.zeros((1, 21))
    cells[0, 1:7] = [0, 0, 5, 1, 0, 0]
    cells[0, 13], cells[0, 14] = 1.0, 0.5
    o = orc.Oracle(params(1e-4, M0=0.0))
    o.set_cells(cells)
    o.loop_init()
    with pytest.raises(RuntimeError, match="cell mass"):
        o.iterate(1)
