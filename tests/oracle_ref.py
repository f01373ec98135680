"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle_abm.so) for the tests.

The oracle is test infrastructure: a C++ restatement of the reference's 3-D
mechanics step (see oracle/abm3d.hpp).  Here it is only what results are compared against.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "liboracle_abm.so")


def build_oracle():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("R", ctypes.c_double), ("Rcell", ctypes.c_double), ("E0", ctypes.c_double),
        ("Ecell", ctypes.c_double), ("L0", ctypes.c_double), ("Ldiv", ctypes.c_double),
        ("neighbor_threshold", ctypes.c_double), ("nz_threshold", ctypes.c_double),
        ("adhesion_mode", ctypes.c_int), ("integration_mode", ctypes.c_int),
        ("max_stepsize", ctypes.c_double), ("min_stepsize", ctypes.c_double),
        ("max_error_allowed", ctypes.c_double), ("min_error", ctypes.c_double),
        ("max_tries_update_stepsize", ctypes.c_int), ("iter_update_stepsize", ctypes.c_int),
        ("iter_update_neighbors", ctypes.c_int),
        ("max_rxy_noise", ctypes.c_double), ("max_rz_noise", ctypes.c_double),
        ("max_nxy_noise", ctypes.c_double), ("max_nz_noise", ctypes.c_double),
        ("cell_surface_coulomb_coeff", ctypes.c_double), ("no_surface", ctypes.c_int),
        ("growth_mean", ctypes.c_double), ("growth_std", ctypes.c_double),
        ("daughter_length_std", ctypes.c_double), ("daughter_angle_xy_bound", ctypes.c_double),
        ("daughter_angle_z_bound", ctypes.c_double), ("rng_seed", ctypes.c_ulonglong),
        ("n_start_multithread", ctypes.c_int), ("n_threads", ctypes.c_int),
        ("friction_mode", ctypes.c_int), ("cell_cell_coulomb_coeff", ctypes.c_double),
        ("M0", ctypes.c_double), ("controller", ctypes.c_int),
    ]


def _load():
    if not os.path.exists(ORACLE_LIB):
        build_oracle()
    lib = ctypes.CDLL(ORACLE_LIB)
    P = ctypes.POINTER
    d, i, vp, dp, ip = ctypes.c_double, ctypes.c_int, ctypes.c_void_p, P(ctypes.c_double), P(ctypes.c_int)
    sig = {
        "oracle_create": ([P(OracleParams), P(vp)], i),
        "oracle_destroy": ([vp], None),
        "oracle_last_error": ([], ctypes.c_char_p),
        "oracle_max_threads": ([], i),
        "oracle_set_jkr_table": ([vp, dp, dp, i], i),
        "oracle_jkr_table": ([d, d, d, d, i, dp, dp], i),
        "oracle_jkr_contact_radius": ([d, d, d, d], d),
        "oracle_jkr_equilibrium_distance": ([d, d, d, d], d),
        "oracle_jkr_optimal_gamma": ([d, d, d, d], d),
        "oracle_set_cells": ([vp, dp, i, i, i], i),
        "oracle_get_num_cells": ([vp], i),
        "oracle_get_cells": ([vp, dp, i], i),
        "oracle_set_parents": ([vp, ip, i], i),
        "oracle_get_parents": ([vp, ip, i], i),
        "oracle_set_clock": ([vp, d, d, i], None),
        "oracle_get_clock": ([vp, dp, dp, ip], None),
        "oracle_build_neighbors": ([vp], i),
        "oracle_set_cpu_optimized": ([vp, i], None),
        "oracle_set_rng_stream": ([vp, i, ctypes.c_uint], None),
        "oracle_rng_stream_draws": ([vp], ctypes.c_longlong),
        "oracle_rng_stream_uniforms": ([ctypes.c_uint, i, dp], None),
        "oracle_num_neighbors": ([vp], i),
        "oracle_get_neighbors": ([vp, dp, i], i),
        "oracle_set_neighbors": ([vp, dp, i, i], i),
        "oracle_update_neighbor_distances": ([vp], i),
        "oracle_dist_between_cells": ([dp, dp, d, dp, dp, d, dp], None),
        "oracle_nearest_body_coord": ([dp, dp, d, dp], d),
        "oracle_cell_cell_forces": ([vp, dp], i),
        "oracle_conservative_forces": ([vp, dp], i),
        "oracle_get_velocities": ([vp, dp], i),
        "oracle_rk_attempt": ([vp, d, i, i, dp, dp, dp], i),
        "oracle_loop_init": ([vp], i),
        "oracle_iterate": ([vp, i, i, i], i),
        "oracle_get_stats": ([vp, P(ctypes.c_longlong), P(ctypes.c_longlong), P(ctypes.c_longlong), dp], None),
        "oracle_rejected": ([vp], ctypes.c_longlong),
        "oracle_grow": ([vp, d], i),
        "oracle_divide": ([vp, d, i], i),
        "oracle_min_dist_to_cell": ([vp, i], d),
        "oracle_rng_uniform": ([ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                ctypes.c_uint, ctypes.c_uint], d),
        "oracle_area_integrals": ([d, d, d, d, dp], None),
        "oracle_integral1": ([d, d, d, d, d, d], d),
        "oracle_integral2": ([d, d, d, d, d, d], d),
        "oracle_integral4": ([d, d, d], d),
        "oracle_integral5": ([d, d, d], d),
        "oracle_integral6": ([d, d, d], d),
        "oracle_surface_forces": ([i, d, d, d, d, d, d, d, d, i, dp], i),
        "oracle_det_log": ([d], d),
        "oracle_jkr_table2": ([d, d, d, d, i, i, dp, dp, dp], i),
        "oracle_set_jkr_table2": ([vp, dp, i, dp, i, dp], i),
        "oracle_set_switching": ([vp, i, i, dp, dp, dp, d, i, ip, dp, d, i, dp, i], i),
        "oracle_set_basal": ([vp, i, d], i),
        "oracle_switch_markov": ([vp, d, i], i),
        "oracle_switch_inherit": ([vp, ip, i, i], i),
        "oracle_switch_ramps": ([vp, d], i),
        "oracle_basal_compact": ([vp], i),
        "oracle_det_sincos": ([d, dp, dp], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


LIB = _load()


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def dist_between_cells(r1, n1, h1, r2, n2, h2):
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (r1, n1, r2, n2)]
    out = np.zeros(5)
    LIB.oracle_dist_between_cells(_dp(a[0]), _dp(a[1]), h1, _dp(a[2]), _dp(a[3]), h2, _dp(out))
    return out[:3], out[3], out[4]


def nearest_body_coord(r, n, h, q):
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (r, n, q)]
    return LIB.oracle_nearest_body_coord(_dp(a[0]), _dp(a[1]), h, _dp(a[2]))


def jkr_table_variable(R, Rcell, E0, max_gamma, n_delta=100, n_gamma=100):
    """(overlap mesh, gamma mesh, radii (n_delta, n_gamma)) of simulation.hpp:120-145."""
    d, g = np.zeros(n_delta), np.zeros(n_gamma)
    r = np.zeros(n_delta * n_gamma)
    LIB.oracle_jkr_table2(R, Rcell, E0, max_gamma, n_delta, n_gamma, _dp(d), _dp(g), _dp(r))
    return d, g, r.reshape(n_delta, n_gamma)


def rng_stream_uniforms(seed, k):
    """The first k uniforms of the reference's random source seeded with `seed`."""
    out = np.zeros(k)
    LIB.oracle_rng_stream_uniforms(int(seed), k, _dp(out))
    return out


def jkr_table(R, Rcell, E0, gamma, n_mesh=100):
    d, r = np.zeros(n_mesh), np.zeros(n_mesh)
    LIB.oracle_jkr_table(R, Rcell, E0, gamma, n_mesh, _dp(d), _dp(r))
    return d, r


class Oracle:
    """The oracle's loop state; parameters use the same names as abm_b200.DEFAULTS."""

    def __init__(self, pdict, jkr=None, n_threads=0, n_start_multithread=50, cpu_optimized=False):
        """cpu_optimized: the cell-list neighbor build and OpenMP over the pairs (the
        "optimized CPU" context figure), in place of the reference's procedures."""
        p = OracleParams()
        for name, _ in OracleParams._fields_:
            if name in pdict:
                setattr(p, name, pdict[name])
        p.n_start_multithread = n_start_multithread
        p.n_threads = n_threads
        self.pdict = dict(pdict)
        self._c = ctypes.c_void_p()
        LIB.oracle_create(ctypes.byref(p), ctypes.byref(self._c))
        LIB.oracle_set_cpu_optimized(self._c, 1 if cpu_optimized else 0)
        if jkr is not None:
            self.set_jkr_table(*jkr)
        self.ncols = None

    def __del__(self):
        if getattr(self, "_c", None):
            LIB.oracle_destroy(self._c)
            self._c = None

    def set_jkr_table_variable(self, delta, gamma, radius):
        d = np.ascontiguousarray(delta, dtype=np.float64)
        g = np.ascontiguousarray(gamma, dtype=np.float64)
        r = np.ascontiguousarray(radius, dtype=np.float64).ravel()
        LIB.oracle_set_jkr_table2(self._c, _dp(d), len(d), _dp(g), len(g), _dp(r))

    def set_switching(self, mode=1, rates=(0.0, 0.0, 0.0, 0.0), growth=((0.0, 0.0), (0.0, 0.0)), timescale=0.0,
                      attrs=(), max_gamma=0.0, modulate=0, visc=(0.0, 0.0, 0.0, 0.0), max_coord=1, n_start=0):
        """oracle_set_switching with the arguments of Simulation.set_switching."""
        cols = (ctypes.c_int * 4)(*[int(c) for c, _, _ in attrs])
        targets = np.array([t1 for _, t1, _ in attrs] + [t2 for _, _, t2 in attrs] + [0.0], dtype=np.float64)
        rc = LIB.oracle_set_switching(self._c, int(mode), int(n_start), _dp(np.array(rates, dtype=np.float64)),
                                      _dp(np.array(growth[0], dtype=np.float64)),
                                      _dp(np.array(growth[1], dtype=np.float64)), float(timescale), len(attrs), cols,
                                      _dp(targets), float(max_gamma), int(modulate),
                                      _dp(np.array(visc, dtype=np.float64)), int(max_coord))
        assert rc == 0

    def set_basal_only(self, on=True, min_overlap=0.0):
        LIB.oracle_set_basal(self._c, int(bool(on)), float(min_overlap))

    def set_jkr_table(self, delta, radius):
        d = np.ascontiguousarray(delta, dtype=np.float64)
        r = np.ascontiguousarray(radius, dtype=np.float64)
        LIB.oracle_set_jkr_table(self._c, _dp(d), _dp(r), len(d))

    def set_cells(self, cells):
        a = np.asfortranarray(cells, dtype=np.float64)
        LIB.oracle_set_cells(self._c, _dp(a), a.shape[0], a.shape[1], a.shape[0])
        self.ncols = a.shape[1]

    def cells(self):
        n = LIB.oracle_get_num_cells(self._c)
        out = np.zeros((n, self.ncols), order="F")
        LIB.oracle_get_cells(self._c, _dp(out), max(n, 1))
        return out

    def set_clock(self, t, dt, iteration):
        LIB.oracle_set_clock(self._c, t, dt, iteration)

    def clock(self):
        t, dt, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        LIB.oracle_get_clock(self._c, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it))
        return t.value, dt.value, it.value

    def set_parents(self, parents):
        a = np.ascontiguousarray(parents, dtype=np.int32)
        LIB.oracle_set_parents(self._c, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(a))

    def parents(self):
        n = LIB.oracle_get_parents(self._c, None, 0)
        a = np.zeros(n, dtype=np.int32)
        LIB.oracle_get_parents(self._c, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n)
        return a

    def build_neighbors(self):
        return LIB.oracle_build_neighbors(self._c)

    def neighbors(self):
        m = LIB.oracle_num_neighbors(self._c)
        out = np.zeros((m, 7), order="F")
        LIB.oracle_get_neighbors(self._c, _dp(out), max(m, 1))
        return out

    def set_neighbors(self, rows):
        a = np.asfortranarray(rows, dtype=np.float64)
        LIB.oracle_set_neighbors(self._c, _dp(a), a.shape[0], max(a.shape[0], 1))

    def update_neighbor_distances(self):
        LIB.oracle_update_neighbor_distances(self._c)

    def _n6(self, fn):
        n = LIB.oracle_get_num_cells(self._c)
        out = np.zeros((n, 6), order="F")
        if fn(self._c, _dp(out)):
            raise RuntimeError(LIB.oracle_last_error().decode())
        return out

    def cell_cell_forces(self):
        return self._n6(LIB.oracle_cell_cell_forces)

    def conservative_forces(self):
        return self._n6(LIB.oracle_conservative_forces)

    def get_velocities(self):
        return self._n6(LIB.oracle_get_velocities)

    def rk_attempt(self, dt, iteration=0, attempt=0):
        n = LIB.oracle_get_num_cells(self._c)
        cells = np.zeros((n, self.ncols), order="F")
        errors = np.zeros((n, 6), order="F")
        e = ctypes.c_double()
        if LIB.oracle_rk_attempt(self._c, dt, iteration, attempt, _dp(cells), _dp(errors), ctypes.byref(e)):
            raise RuntimeError(LIB.oracle_last_error().decode())
        return cells, errors, e.value

    def loop_init(self):
        return LIB.oracle_loop_init(self._c)

    def iterate(self, n_iters, n_cells=0, fast_cc=1):
        rc = LIB.oracle_iterate(self._c, n_iters, n_cells, fast_cc)
        if rc:
            raise RuntimeError(LIB.oracle_last_error().decode())

    def stats(self):
        a, r, dv = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        e = ctypes.c_double()
        LIB.oracle_get_stats(self._c, ctypes.byref(a), ctypes.byref(r), ctypes.byref(dv), ctypes.byref(e))
        return dict(attempts=a.value, rebuilds=r.value, divisions=dv.value, last_max_error=e.value,
                    rejected=LIB.oracle_rejected(self._c))

    def grow(self, dt):
        LIB.oracle_grow(self._c, dt)

    def divide(self, t, iteration):
        return LIB.oracle_divide(self._c, t, iteration)

    def set_rng_stream(self, seed):
        """Draw every random number from one mt19937 seeded with `seed`, in the reference's
        order (simulation.hpp:1173), instead of the Philox counter policy; None: Philox."""
        LIB.oracle_set_rng_stream(self._c, 0 if seed is None else 1, 0 if seed is None else int(seed))

    def rng_stream_draws(self):
        return LIB.oracle_rng_stream_draws(self._c)

    def min_dist_to_cell(self, i):
        return LIB.oracle_min_dist_to_cell(self._c, i)


# ---------------------------------------------------------------------------
# 2-D restatement (oracle/abm2d.hpp, oracle/capi2d.cpp)
# ---------------------------------------------------------------------------
class Oracle2DParams(ctypes.Structure):
    _fields_ = [
        ("R", ctypes.c_double), ("Rcell", ctypes.c_double), ("E0", ctypes.c_double),
        ("Ecell", ctypes.c_double), ("sigma0", ctypes.c_double), ("Ldiv", ctypes.c_double),
        ("neighbor_threshold", ctypes.c_double), ("adhesion_mode", ctypes.c_int),
        ("adhesion_strength", ctypes.c_double), ("adhesion_mindist", ctypes.c_double),
        ("integration_mode", ctypes.c_int), ("max_stepsize", ctypes.c_double),
        ("min_stepsize", ctypes.c_double), ("max_error_allowed", ctypes.c_double),
        ("min_error", ctypes.c_double), ("max_tries_update_stepsize", ctypes.c_int),
        ("iter_update_stepsize", ctypes.c_int), ("iter_update_neighbors", ctypes.c_int),
        ("max_noise", ctypes.c_double), ("growth_mean", ctypes.c_double), ("growth_std", ctypes.c_double),
        ("daughter_length_std", ctypes.c_double), ("daughter_angle_bound", ctypes.c_double),
        ("rng_seed", ctypes.c_ulonglong), ("use_pf", ctypes.c_int), ("pf", ctypes.c_double * 3),
    ]


def _load2d(lib):
    P = ctypes.POINTER
    d, i, vp, dp, ip = ctypes.c_double, ctypes.c_int, ctypes.c_void_p, P(ctypes.c_double), P(ctypes.c_int)
    ll = P(ctypes.c_longlong)
    sig = {
        "oracle2d_create": ([P(Oracle2DParams), P(vp)], i),
        "oracle2d_destroy": ([vp], None),
        "oracle2d_set_cells": ([vp, dp, i, i, i], i),
        "oracle2d_get_num_cells": ([vp], i),
        "oracle2d_get_cells": ([vp, dp, i], i),
        "oracle2d_set_parents": ([vp, ip, i], i),
        "oracle2d_get_parents": ([vp, ip, i], i),
        "oracle2d_set_clock": ([vp, d, d, i], None),
        "oracle2d_get_clock": ([vp, dp, dp, ip], None),
        "oracle2d_build_neighbors": ([vp], i),
        "oracle2d_num_neighbors": ([vp], i),
        "oracle2d_get_neighbors": ([vp, dp, i, ip], i),
        "oracle2d_cell_cell_forces": ([vp, dp], i),
        "oracle2d_get_velocities": ([vp, dp], i),
        "oracle2d_rk_attempt": ([vp, d, i, i, dp, dp, dp], i),
        "oracle2d_loop_init": ([vp], i),
        "oracle2d_iterate": ([vp, i, i], i),
        "oracle2d_get_stats": ([vp, ll, ll, ll, dp], None),
        "oracle2d_divide": ([vp, d, i, ip], i),
        "oracle2d_set_rng_stream": ([vp, i, ctypes.c_uint], None),
        "oracle2d_rng_stream_draws": ([vp], ctypes.c_longlong),
        "oracle2d_grow": ([vp, d], i),
        "oracle2d_jkr_lagrange_pair": ([dp, dp, dp, d, d, d, d, dp], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res


_load2d(LIB)


def jkr_lagrange_pair(n1, n2, d12, R, s, t, dmin):
    """forcesJKRLagrange (2D/include/adhesion.hpp:403-448) with the constraint: 2 x 4 dE/dq."""
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (n1, n2, d12)]
    out = np.zeros(8)
    LIB.oracle2d_jkr_lagrange_pair(_dp(a[0]), _dp(a[1]), _dp(a[2]), R, s, t, dmin, _dp(out))
    return out.reshape(2, 4)


class Oracle2D:
    """The 2-D oracle; parameter names as abm_b200.DEFAULTS (max_noise, sigma0, adhesion_*)."""

    def __init__(self, pdict, pf=None):
        import abm_b200
        full = dict(abm_b200.DEFAULTS)
        full.update(abm_b200.DEFAULTS_2D)
        full.update(pdict)
        pdict = full
        p = Oracle2DParams()
        for name, _ in Oracle2DParams._fields_:
            if name in pdict and name not in ("pf", "use_pf"):
                setattr(p, name, pdict[name])
        p.daughter_angle_bound = pdict.get("daughter_angle_xy_bound", 0.0)
        if pf is not None:
            p.use_pf = 1
            for k in range(3):
                p.pf[k] = pf[k]
        self._c = ctypes.c_void_p()
        LIB.oracle2d_create(ctypes.byref(p), ctypes.byref(self._c))
        self.ncols = None

    def __del__(self):
        if getattr(self, "_c", None):
            LIB.oracle2d_destroy(self._c)
            self._c = None

    def set_cells(self, cells):
        a = np.asfortranarray(cells, dtype=np.float64)
        self.ncols = a.shape[1]
        LIB.oracle2d_set_cells(self._c, _dp(a), a.shape[0], a.shape[1], max(a.shape[0], 1))

    def cells(self):
        n = LIB.oracle2d_get_num_cells(self._c)
        out = np.zeros((n, self.ncols), order="F")
        LIB.oracle2d_get_cells(self._c, _dp(out), max(n, 1))
        return out

    def set_parents(self, parents):
        a = np.ascontiguousarray(parents, dtype=np.int32)
        LIB.oracle2d_set_parents(self._c, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(a))

    def parents(self):
        n = LIB.oracle2d_get_parents(self._c, None, 0)
        a = np.zeros(n, dtype=np.int32)
        LIB.oracle2d_get_parents(self._c, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n)
        return a

    def set_clock(self, t, dt, iteration):
        LIB.oracle2d_set_clock(self._c, t, dt, iteration)

    def clock(self):
        t, dt, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        LIB.oracle2d_get_clock(self._c, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it))
        return t.value, dt.value, it.value

    def build_neighbors(self):
        return LIB.oracle2d_build_neighbors(self._c)

    def neighbors(self, with_adhere=False):
        m = LIB.oracle2d_num_neighbors(self._c)
        out = np.zeros((m, 6), order="F")
        adh = np.zeros(max(m, 1), dtype=np.int32)
        LIB.oracle2d_get_neighbors(self._c, _dp(out), max(m, 1), adh.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return (out, adh[:m]) if with_adhere else out

    def _n4(self, fn):
        n = LIB.oracle2d_get_num_cells(self._c)
        out = np.zeros((n, 4), order="F")
        fn(self._c, _dp(out))
        return out

    def cell_cell_forces(self):
        return self._n4(LIB.oracle2d_cell_cell_forces)

    def get_velocities(self):
        return self._n4(LIB.oracle2d_get_velocities)

    def rk_attempt(self, dt, iteration=0, attempt=0):
        n = LIB.oracle2d_get_num_cells(self._c)
        cells = np.zeros((n, self.ncols), order="F")
        errors = np.zeros((n, 4), order="F")
        e = ctypes.c_double()
        LIB.oracle2d_rk_attempt(self._c, dt, iteration, attempt, _dp(cells), _dp(errors), ctypes.byref(e))
        return cells, errors, e.value

    def loop_init(self):
        return LIB.oracle2d_loop_init(self._c)

    def iterate(self, n_iters, n_cells=0):
        return LIB.oracle2d_iterate(self._c, n_iters, n_cells)

    def stats(self):
        a, r, dv = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        e = ctypes.c_double()
        LIB.oracle2d_get_stats(self._c, ctypes.byref(a), ctypes.byref(r), ctypes.byref(dv), ctypes.byref(e))
        return dict(attempts=a.value, rebuilds=r.value, divisions=dv.value, last_max_error=e.value)

    def divide(self, t, iteration):
        tr = ctypes.c_int()
        nd = LIB.oracle2d_divide(self._c, t, iteration, ctypes.byref(tr))
        return nd, tr.value

    def set_rng_stream(self, seed):
        """The reference's sequential mt19937 source seeded with `seed`; None: Philox."""
        LIB.oracle2d_set_rng_stream(self._c, 0 if seed is None else 1, 0 if seed is None else int(seed))

    def rng_stream_draws(self):
        return LIB.oracle2d_rng_stream_draws(self._c)
    def grow(self, dt):
        LIB.oracle2d_grow(self._c, dt)
