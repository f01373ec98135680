"""The oracle's cell-surface forces (mechanics.hpp:673-780 and :800-910, restated in
oracle/abm3d.hpp) pinned the way the reference's own tests pin them
(ABM-3d/ABM-3d-cpp/test/src/testCellSurfaceRepulsionForces.cpp and
testCellSurfaceAdhesionForces.cpp): for ten orientations nz = sin(pi/2 (i + 1) / 10), a
cell overlapping the surface by at most 0.2 R and a cell 0.1 R clear of it, the z and
nz forces equal the derivatives of the surface energies with respect to rz and nz, and
the other four forces are zero.

  repulsion  E = E0 sqrt(R) (R^-1/2 (1 - nz^2) I1(2) + 4/3 nz^2 I1(3/2))
             (testCellSurfaceRepulsionForces.cpp:43-80, I1(g) = integral1 with exponent g)
  adhesion   E = -sigma0 areaIntegral1   (testCellSurfaceAdhesionForces.cpp:41-60)

The reference differentiates in 100-digit MPFR with a step of 1e-50; in doubles a
Richardson-extrapolated central difference stands in, so the bar is a relative 1e-8
instead of an absolute 1e-45.  The horizontal branch (nz below the threshold) is checked
against its closed forms and against the tilted branch at a small nz, and the single-cell
conservative forces against the sum of both energies (testConservativeForces.cpp)."""
import ctypes
import math

import numpy as np
import pytest

import oracle_ref as orc

R = 0.8
E0 = 3900.0
SIGMA0 = 100.0
HALF_L = 0.5
NZ_THRESHOLD = 1e-8
ANGLES = [math.pi / 2 * (i + 1) / 10 for i in range(10)]
CASES = {"contact": 0.2 * R, "clear": -0.1 * R}       # maximum overlap of the cell
REL = 1e-8


def forces(kind, rz, angle=None, nz=None, half_l=HALF_L):
    if nz is None:
        nz = math.sin(angle)
    nx = math.cos(angle) if angle is not None else math.sqrt(max(0.0, 1 - nz * nz))
    out = np.zeros(6)
    rc = orc.LIB.oracle_surface_forces(kind, rz, nx, nz, half_l, SIGMA0, R, E0, NZ_THRESHOLD, 0,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0
    return out


def i1(rz, nz, gamma):
    return orc.LIB.oracle_integral1(rz, nz, R, HALF_L, gamma, (R - rz) / nz)


def repulsion_energy(rz, nz):
    return E0 * math.sqrt(R) * (R ** -0.5 * (1 - nz * nz) * i1(rz, nz, 2.0) + 4.0 / 3.0 * nz * nz * i1(rz, nz, 1.5))


def adhesion_energy(rz, nz):
    area = np.zeros(3)
    orc.LIB.oracle_area_integrals(rz, nz, R, HALF_L, area.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return -SIGMA0 * area[0]


def derivative(f, x, h=1e-4):
    """Central difference with one Richardson step (error O(h^4))."""
    d1 = (f(x + h) - f(x - h)) / (2 * h)
    d2 = (f(x + h / 2) - f(x - h / 2)) / h
    return (4 * d2 - d1) / 3


ENERGY = {0: repulsion_energy, 1: adhesion_energy}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("kind", [0, 1], ids=["repulsion", "adhesion"])
def test_surface_forces_are_energy_derivatives(kind, case):
    energy = ENERGY[kind]
    for angle in ANGLES:
        nz = math.sin(angle)
        rz = R + HALF_L * nz - CASES[case]     # testCellSurfaceRepulsionForces.cpp:107-108, :150-151
        f = forces(kind, rz, angle)
        assert f[0] == 0 and f[1] == 0 and f[3] == 0 and f[4] == 0
        if case == "clear":
            assert f[2] == 0 and f[5] == 0
            continue
        d_rz = derivative(lambda x: energy(x, nz), rz)
        d_nz = derivative(lambda x: energy(rz, x), nz)
        scale = max(abs(d_rz), abs(d_nz), 1.0)
        assert abs(f[2] - d_rz) < REL * scale, (angle, f[2], d_rz)
        assert abs(f[5] - d_nz) < REL * scale, (angle, f[5], d_nz)
        assert abs(f[2]) > 1.0                 # the cell really is pressed into / held by the surface


@pytest.mark.parametrize("kind", [0, 1], ids=["repulsion", "adhesion"])
def test_horizontal_branch(kind):
    """nz below the threshold: E_rep = E0 l (R - rz)^2 and E_adh = -sigma0 sqrt(R) l sqrt(R - rz)
    (mechanics.hpp:717-721, :842-846), the nz -> 0 limits of the tilted forms."""
    length = 2 * HALF_L
    for depth in (0.01, 0.05, 0.16):
        rz = R - depth
        f = forces(kind, rz, nz=0.0)
        expect = -2 * E0 * depth * length if kind == 0 else SIGMA0 * math.sqrt(R) * length / (2 * math.sqrt(depth))
        assert abs(f[2] - expect) <= 1e-12 * abs(expect)
        assert f[5] == 0 and f[0] == f[1] == f[3] == f[4] == 0
        tilted = forces(kind, rz, nz=1e-6)     # above the threshold: the general branch
        assert abs(tilted[2] - expect) < REL * abs(expect), (depth, tilted[2], expect)
    assert np.all(forces(kind, R + 0.01, nz=0.0) == 0)   # a horizontal cell clear of the surface


def test_conservative_forces_of_a_single_cell():
    """getConservativeForces for one cell and no neighbors (testConservativeForces.cpp:80-163):
    eleven orientations from horizontal to vertical, each overlapping the surface by 0.2 R.
    The x, y forces and torques are zero; the z force and nz torque are minus the
    derivatives of the repulsion plus adhesion energies, and for the horizontal cell
    2 E0 (R - rz) l - sigma0 sqrt(R) l / (2 sqrt(R - rz)) and 0."""
    import abm_b200
    _, p = abm_b200.make_params(adhesion_mode=0, nz_threshold=NZ_THRESHOLD, no_surface=0)
    p["R"], p["E0"] = R, E0
    total = lambda rz, nz: repulsion_energy(rz, nz) + adhesion_energy(rz, nz)
    for j in range(11):
        angle = math.pi / 2 * j / 10
        nz = math.sin(angle)
        rz = R + HALF_L * nz - 0.2 * R
        cells = np.zeros((1, 21))
        cells[0, 3:7] = [rz, math.cos(angle), 0.0, nz]
        cells[0, 13], cells[0, 14], cells[0, 19] = 2 * HALF_L, HALF_L, SIGMA0
        o = orc.Oracle(p)
        o.set_cells(cells)
        o.build_neighbors()
        f = o.conservative_forces()[0]
        assert f[0] == 0 and f[1] == 0 and f[3] == 0 and f[4] == 0
        if nz > 0:
            target = (-derivative(lambda x: total(x, nz), rz), -derivative(lambda x: total(rz, x), nz))
        else:
            depth, length = R - rz, 2 * HALF_L
            target = (2 * E0 * depth * length - 0.5 * SIGMA0 * math.sqrt(R) * length / math.sqrt(depth), 0.0)
        scale = max(abs(target[0]), abs(target[1]), 1.0)
        assert abs(f[2] - target[0]) < REL * scale, (angle, f[2], target[0])
        assert abs(f[5] - target[1]) < REL * scale, (angle, f[5], target[1])
