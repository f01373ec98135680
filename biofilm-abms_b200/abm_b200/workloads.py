"""Seeded synthetic biofilm states in the reference's cell-array layout.

`biofilm_3d` draws the 100k-cell 3-D benchmark state: centres uniform in a
disk of radius 300 um with z in [R, 10] um, azimuth uniform on [0, 2 pi),
polar angle from the substrate uniform on [0, pi/2], lengths uniform on
[2, 5] um.  Pairs whose centrelines come closer than `min_gap` (default
2 Rcell + 0.1 um, i.e. no overlap reaching the hard cell cores) are resolved
by redrawing one cell of the pair, so every initial contact lies in the EPS
shell; `contact_boost` then moves a fraction of cells into contact with a
random neighbour (overlap drawn uniformly in the EPS shell) to raise the mean
contact count.  All draws come from numpy's PCG64 seeded with `seed`.
"""
import ctypes

import numpy as np

NCOLS_3D = 22   # indices.hpp:17-47 plus gamma (column 21)
NCOLS_2D = 17   # ABM-2d/ABM-2d-cpp/include/indices.hpp:17-41


def _host_lib(lib):
    """The library that holds the generator: this package's, unless another build of
    csrc/abm_workload.cpp (a ctypes handle) is given."""
    if lib is not None:
        return lib
    from . import LIB
    return LIB


def _generate(n, seed, disk_radius, z_lo, z_hi, lmin, lmax, min_gap, contact_dist, p_contact,
              max_tries=10000, lib=None):
    LIB = _host_lib(lib)
    LIB.abm_generate_biofilm_3d.argtypes = [
        ctypes.c_int, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    LIB.abm_generate_biofilm_3d.restype = ctypes.c_int
    r = np.zeros((n, 3))
    nv = np.zeros((n, 3))
    l = np.zeros(n)
    placed = ctypes.c_int()
    rc = LIB.abm_generate_biofilm_3d(n, seed, disk_radius, z_lo, z_hi, lmin, lmax, min_gap, contact_dist,
                                     p_contact, max_tries, r.ctypes.data, nv.ctypes.data, l.ctypes.data,
                                     ctypes.byref(placed))
    if rc:
        raise RuntimeError("could only place %d of %d cells" % (placed.value, n))
    return r, nv, l


def count_close_pairs(cells, dist, lmax=None, lib=None):
    """Number of unordered pairs with centreline distance < dist."""
    LIB = _host_lib(lib)
    LIB.abm_count_close_pairs_3d.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
    LIB.abm_count_close_pairs_3d.restype = ctypes.c_longlong
    r = np.ascontiguousarray(cells[:, 1:4])
    nv = np.ascontiguousarray(cells[:, 4:7])
    l = np.ascontiguousarray(cells[:, 13])
    lmax = float(l.max()) if lmax is None else lmax
    return int(LIB.abm_count_close_pairs_3d(len(l), r.ctypes.data, nv.ctypes.data, l.ctypes.data, dist, lmax))


def biofilm_3d(n=100_000, seed=1, disk_radius=300.0, z_max=10.0, R=0.8, Rcell=0.5,
               lmin=2.0, lmax=5.0, eta0=100.0, eta1=720.0, sigma0=100.0, gamma=100.0,
               growth=0.0, min_gap=None, p_contact=0.0, lib=None):
    """Return an (n, 22) float64 cell array (Fortran order) and a summary dict.  `lib`:
    another build of the generator to draw with (default: this package's library)."""
    gap = 2 * Rcell + 0.1 if min_gap is None else min_gap
    r, nv, l = _generate(n, seed, disk_radius, R, z_max, lmin, lmax, gap, 2 * R, p_contact, lib=lib)
    cells = np.zeros((n, NCOLS_3D), dtype=np.float64, order="F")
    cells[:, 0] = np.arange(n)
    cells[:, 1:4] = r
    cells[:, 4:7] = nv
    cells[:, 13] = l
    cells[:, 14] = l / 2
    cells[:, 16] = growth
    cells[:, 17] = eta0
    cells[:, 18] = eta1
    cells[:, 19] = sigma0
    cells[:, 20] = 1
    cells[:, 21] = gamma
    contacts = count_close_pairs(cells, 2 * R, lmax, lib=lib)
    info = dict(n=n, seed=seed, min_gap=gap, p_contact=p_contact,
                mean_contacts_per_cell=2.0 * contacts / n)
    return cells, info


def two_cell_3d(r1, n1, r2, n2, half_l=0.5, eta0=100.0, eta1=720.0, sigma0=100.0, gamma=100.0):
    """Two cells in the layout of testTwoCellSimulations.cpp:91-96 (plus gamma)."""
    cells = np.zeros((2, NCOLS_3D), dtype=np.float64, order="F")
    for k, (r, n) in enumerate(((r1, n1), (r2, n2))):
        cells[k, 0] = k
        cells[k, 1:4] = r
        cells[k, 4:7] = n
        cells[k, 13] = 2 * half_l
        cells[k, 14] = half_l
        cells[k, 17] = eta0
        cells[k, 18] = eta1
        cells[k, 19] = sigma0
        cells[k, 20] = 1
        cells[k, 21] = gamma
    return cells


def founder_3d(L0=2.0, R=0.8, E0=3900.0, sigma0=100.0, growth=1.5, eta0=100.0, eta1=720.0, gamma=100.0):
    """One cell at the origin along (1, 0, 0) resting on the surface at the height
    rz = R - (sigma0 sqrt(R) / (4 E0))^(2/3), with centreline length L0 and the mean
    growth rate (the 3-D driver's start, abmConstAdhesion.cpp:414-431)."""
    cells = np.zeros((1, NCOLS_3D), dtype=np.float64, order="F")
    cells[0, 3] = R - (sigma0 * np.sqrt(R) / (4 * E0)) ** (2.0 / 3.0)
    cells[0, 4] = 1.0
    cells[0, 13] = L0
    cells[0, 14] = L0 / 2
    cells[0, 16] = growth
    cells[0, 17] = eta0
    cells[0, 18] = eta1
    cells[0, 19] = sigma0
    cells[0, 20] = 1
    cells[0, 21] = gamma
    return cells


def biofilm_2d(n, seed=1, disk_radius=None, lmin=2.0, lmax=4.4, R=0.8, Rcell=0.5, eta0=100.0, eta1=100.0,
               growth=0.0, min_gap=None, p_contact=0.9, density=0.1):
    """A seeded 2-D colony in the 17-column layout of ABM-2d/ABM-2d-cpp/include/indices.hpp:
    centres uniform in a disk (radius from `density` cells per um^2 unless given),
    orientations uniform in the plane, lengths uniform on [lmin, lmax], contacts
    inside the EPS shell as in biofilm_3d."""
    from . import LIB
    gap = 2 * Rcell + 0.1 if min_gap is None else min_gap
    if disk_radius is None:
        disk_radius = float(np.sqrt(n / (np.pi * density)))
    LIB.abm_generate_biofilm_2d.argtypes = [
        ctypes.c_int, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.POINTER(ctypes.c_int)]
    LIB.abm_generate_biofilm_2d.restype = ctypes.c_int
    r = np.zeros((n, 3))
    nv = np.zeros((n, 3))
    l = np.zeros(n)
    placed = ctypes.c_int()
    rc = LIB.abm_generate_biofilm_2d(n, seed, disk_radius, lmin, lmax, gap, 2 * R, p_contact, 10000,
                                     r.ctypes.data, nv.ctypes.data, l.ctypes.data, ctypes.byref(placed))
    if rc:
        raise RuntimeError("could only place %d of %d cells" % (placed.value, n))
    cells = np.zeros((n, NCOLS_2D), dtype=np.float64, order="F")
    cells[:, 0] = np.arange(n)
    cells[:, 1:3] = r[:, :2]
    cells[:, 3:5] = nv[:, :2]
    cells[:, 9] = l
    cells[:, 10] = l / 2
    cells[:, 12] = growth
    cells[:, 13] = eta0
    cells[:, 14] = eta1
    cells[:, 15] = eta1
    return cells


def founder_2d(L0=2.0, growth=1.5, eta0=100.0, eta1=100.0):
    """One cell at the origin along (1, 0) with centreline length L0 (the 2-D driver's start)."""
    cells = np.zeros((1, NCOLS_2D), dtype=np.float64, order="F")
    cells[0, 3] = 1.0
    cells[0, 9] = L0
    cells[0, 10] = L0 / 2
    cells[0, 12] = growth
    cells[0, 13] = eta0
    cells[0, 14] = eta1
    cells[0, 15] = eta1
    return cells
