"""Python binding of the B200 mechanics step (ctypes over include/abm_capi.h).

The names mirror the reference functions the C ABI stands in for
(kmnam/biofilm-ABMs, ABM-3d/ABM-3d-cpp/include):

    Simulation.get_cell_neighbors()        getCellNeighbors          mechanics.hpp:520-593
    Simulation.neighbors()                 the neighbor table after updateNeighborDistances (:604-648)
    Simulation.cell_cell_forces()          cellCellInteractionForces mechanics.hpp:1209-1659
    Simulation.get_velocities()            getVelocities             mechanics.hpp:2011-2347
    Simulation.step_runge_kutta_adaptive() stepRungeKuttaAdaptive    mechanics.hpp:2406-2612
    Simulation.grow_cells()                growCells                 growth.hpp:51-57
    Simulation.iterate()                   runSimulation loop body   simulation.hpp:1617-1864

Arrays use the reference layout: cells are (n, ncols) float64 with the column
order of indices.hpp (column 21 = gamma when adhesion is on); neighbor rows
are (m, 7) = (i, j, dx, dy, dz, si, sj).  Errors raise RuntimeError, like the
reference's std::runtime_error.  There is no CPU fallback: the library is
loaded on the first call that needs it (parameter structs, defaults and the
workload helpers need none), and that call raises ImportError when the
library is not built.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libabm_b200.so")

ABM_OK = 0
ERRORS = {-1: "ABM_ERR_ARG", -2: "ABM_ERR_CUDA", -3: "ABM_ERR_CAPACITY", -4: "ABM_ERR_NAN",
          -5: "ABM_ERR_STATE"}
VELOCITY_VERLET, HEUN_EULER, BOGACKI_SHAMPINE, RUNGE_KUTTA_FEHLBERG, DORMAND_PRINCE = 0, 1, 2, 3, 4
PRECISION_FP64, PRECISION_MIXED = 0, 1

# Column indices of the 3-D cell array (ABM-3d/ABM-3d-cpp/include/indices.hpp:17-47)
COL = dict(id=0, rx=1, ry=2, rz=3, nx=4, ny=5, nz=6, drx=7, dry=8, drz=9, dnx=10, dny=11,
           dnz=12, l=13, half_l=14, t0=15, growth=16, eta0=17, eta1=18, sigma0=19, group=20,
           gamma=21)


class AbmParams(ctypes.Structure):
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
        ("precision", ctypes.c_int), ("cap_cells", ctypes.c_int),
        ("cap_neighbors_per_cell", ctypes.c_int), ("pair_lanes", ctypes.c_int),
        ("use_graphs", ctypes.c_int),
        ("controller", ctypes.c_int), ("stepsize_log_capacity", ctypes.c_int),
        ("dims", ctypes.c_int), ("sigma0", ctypes.c_double), ("adhesion_strength", ctypes.c_double),
        ("adhesion_mindist", ctypes.c_double), ("max_noise", ctypes.c_double),
        ("pair_tile", ctypes.c_int), ("pair_blocks_per_sm", ctypes.c_int), ("pair_skin", ctypes.c_double),
        ("pair_sum", ctypes.c_int),
        ("friction_mode", ctypes.c_int), ("cell_cell_coulomb_coeff", ctypes.c_double),
        ("M0", ctypes.c_double),
    ]


class AbmStats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_longlong), ("attempts", ctypes.c_longlong),
        ("retries", ctypes.c_longlong), ("rebuilds", ctypes.c_longlong),
        ("divisions", ctypes.c_longlong), ("t", ctypes.c_double), ("dt", ctypes.c_double),
        ("last_max_error", ctypes.c_double), ("n_cells", ctypes.c_int), ("n_pairs", ctypes.c_int),
        ("rejected", ctypes.c_longlong), ("log_rows", ctypes.c_longlong), ("cell_steps", ctypes.c_longlong),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AbmProfile(ctypes.Structure):
    _fields_ = [
        ("pair_force_ms", ctypes.c_double), ("attempt_ms", ctypes.c_double), ("rebuild_ms", ctypes.c_double),
        ("pair_force_launches", ctypes.c_longlong), ("attempt_launches", ctypes.c_longlong),
        ("rebuild_launches", ctypes.c_longlong), ("iterations", ctypes.c_longlong),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# Defaults: the reference's 3-D driver (ABM-3d/ABM-3d-cpp/src/abmConstAdhesion.cpp) with
# R = 0.8, Rcell = 0.5, E0 = 3900, Ecell = 3.9e6 (testTwoCellSimulations.cpp:46-48),
# L0 = 2 so Ldiv = 2 L0 + 2 R (:41) and neighbor_threshold = 0.5 (2R + Ldiv) (:53).
DEFAULTS = dict(
    R=0.8, Rcell=0.5, E0=3900.0, Ecell=3.9e6, L0=2.0, Ldiv=5.6, neighbor_threshold=3.6,
    nz_threshold=1e-8, adhesion_mode=1, integration_mode=HEUN_EULER, max_stepsize=1e-6,
    min_stepsize=1e-9, max_error_allowed=1e-8, min_error=1e-30, max_tries_update_stepsize=3,
    iter_update_stepsize=1, iter_update_neighbors=100, max_rxy_noise=0.0, max_rz_noise=0.0,
    max_nxy_noise=0.0, max_nz_noise=0.0, cell_surface_coulomb_coeff=1.0, no_surface=0,
    growth_mean=0.0, growth_std=0.0, daughter_length_std=0.0, daughter_angle_xy_bound=0.0,
    daughter_angle_z_bound=0.0, rng_seed=42, precision=PRECISION_FP64, cap_cells=0,
    cap_neighbors_per_cell=0, pair_lanes=8, use_graphs=1, controller=0, stepsize_log_capacity=0,
    dims=3, sigma0=100.0, adhesion_strength=0.0, adhesion_mindist=0.0, max_noise=0.0,
    pair_tile=0, pair_blocks_per_sm=0, pair_skin=0.0, pair_sum=0, friction_mode=0, cell_cell_coulomb_coeff=1.0,
    M0=0.0,
)

# The 2-D driver (ABM-2d/ABM-2d-cpp/include/simulation.hpp:163-237): Bogacki-Shampine 3(2),
# Hertz E0 = 3900 and Ecell = 3.9e6, sigma0 = 100 for the contact density, JKR-Lagrange
# adhesion off unless requested.
DEFAULTS_2D = dict(dims=2, integration_mode=BOGACKI_SHAMPINE, adhesion_mode=0)


def make_params(**kw):
    d = dict(DEFAULTS)
    for k in kw:
        if k not in d:
            raise KeyError("unknown parameter %s" % k)
    d.update(kw)
    p = AbmParams()
    for k, v in d.items():
        setattr(p, k, v)
    return p, d


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("libabm_b200.so is not built (%s); run __graft_entry__.build() or "
                          "make -C biofilm-abms_b200" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    d, i, vp = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
    dp, ip, fp = P(d), P(i), P(ctypes.c_float)
    sig = {
        "abm_create": ([P(AbmParams), P(vp)], i),
        "abm_destroy": ([vp], i),
        "abm_last_error": ([vp], ctypes.c_char_p),
        "abm_get_stream": ([vp, P(vp)], i),
        "abm_synchronize": ([vp], i),
        "abm_jkr_contact_radius": ([d, d, d, d, dp], i),
        "abm_jkr_radius_table": ([d, d, d, d, i, dp, dp], i),
        "abm_jkr_optimal_gamma": ([d, d, d, d, dp], i),
        "abm_set_jkr_table": ([vp, dp, dp, i], i),
        "abm_jkr_radius_table_variable": ([d, d, d, d, i, i, dp, dp, dp], i),
        "abm_set_jkr_table_variable": ([vp, dp, i, dp, i, dp], i),
        "abm_upload_cells": ([vp, dp, i, i, i], i),
        "abm_download_cells": ([vp, dp, i], i),
        "abm_get_num_cells": ([vp, ip], i),
        "abm_set_clock": ([vp, d, d, i], i),
        "abm_get_clock": ([vp, dp, dp, ip], i),
        "abm_set_parents": ([vp, ip, i], i),
        "abm_get_parents": ([vp, ip, i, ip], i),
        "abm_build_neighbors": ([vp, ip], i),
        "abm_download_neighbors": ([vp, dp, i, i, ip], i),
        "abm_upload_neighbors": ([vp, dp, i, i], i),
        "abm_save_checkpoint": ([vp, ctypes.c_char_p], i),
        "abm_load_checkpoint": ([vp, ctypes.c_char_p], i),
        "abm_cell_cell_forces": ([vp, dp], i),
        "abm_get_velocities": ([vp, dp], i),
        "abm_rk_attempt": ([vp, d, i, dp, dp, dp], i),
        "abm_grow": ([vp, d], i),
        "abm_divide": ([vp, ip], i),
        "abm_last_division_tries": ([vp, ip], i),
        "abm_graph_info": ([vp], ctypes.c_char_p),
        "abm_cell_cell_forces_noalloc": ([P(AbmParams), vp, i, i, i, vp, vp, i, dp, dp, i, vp, vp], i),
        "abm_cell_cell_forces_noalloc_status": ([vp], i),
        "abm_noalloc_last_error": ([], ctypes.c_char_p),
        "abm_set_switching": ([vp, i, i, dp, dp, dp, d, i, ip, dp, d, i, dp, i], i),
        "abm_set_basal_only": ([vp, i, d], i),
        "abm_basal_dropped": ([vp, P(ctypes.c_longlong)], i),
        "abm_set_frames": ([vp, d, i], i),
        "abm_frames_taken": ([vp, ip], i),
        "abm_download_frame": ([vp, i, vp, i, ip, dp, ip, ip], i),
        "abm_iterate": ([vp, i, i, P(AbmStats)], i),
        "abm_get_stats": ([vp, P(AbmStats)], i),
        "abm_profile_iterations": ([vp, i, P(AbmProfile)], i),
        "abm_get_adhesion_flags": ([vp, ip, i, ip], i),
        "abm_set_cell_limit": ([vp, i], i),
        "abm_batch_create": ([P(vp), i, P(vp)], i),
        "abm_batch_iterate": ([vp, i], i),
        "abm_batch_synchronize": ([vp], i),
        "abm_batch_get_stream": ([vp, P(vp)], i),
        "abm_batch_destroy": ([vp], i),
        "abm_batch_last_error": ([], ctypes.c_char_p),
        "abm_autotune_pair_tile": ([P(AbmParams), dp, i, i, i, dp, dp, i, i, ip, ip, fp], i),
        "abm_set_adhesion_flags": ([vp, ip, i], i),
        "abm_stepsize_set_weights": ([vp, fp, i], i),
        "abm_stepsize_get_weights": ([vp, fp, i], i),
        "abm_stepsize_get_log": ([vp, fp, i, ip], i),
        "abm_stepsize_clear_log": ([vp], i),
        "abm_mlp_forward": ([fp, fp, i, fp], i),
        "abm_mlp_grad": ([fp, fp, fp, i, fp, fp], i),
        "abm_mlp_train": ([fp, fp, fp, i, i, ctypes.c_float, ctypes.c_uint, fp], i),
        "abm_mlp_last_error": ([], ctypes.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


class _Lib:
    """libabm_b200.so, loaded (with every entry point's signature) on first use."""

    def __init__(self):
        self._lib = None

    def __getattr__(self, name):
        if self._lib is None:
            self._lib = _load()
        return getattr(self._lib, name)


LIB = _Lib()
EXPORTED = ("abm_create abm_destroy abm_last_error abm_get_stream abm_synchronize "
            "abm_jkr_contact_radius abm_jkr_radius_table abm_jkr_optimal_gamma abm_set_jkr_table "
            "abm_jkr_radius_table_variable abm_set_jkr_table_variable abm_upload_cells "
            "abm_download_cells abm_get_num_cells abm_set_clock abm_get_clock abm_set_parents "
            "abm_get_parents abm_build_neighbors abm_download_neighbors abm_upload_neighbors "
            "abm_save_checkpoint abm_load_checkpoint "
            "abm_cell_cell_forces abm_get_velocities abm_rk_attempt abm_grow abm_divide "
            "abm_iterate abm_get_stats abm_profile_iterations abm_last_division_tries abm_graph_info "
            "abm_cell_cell_forces_noalloc abm_cell_cell_forces_noalloc_status abm_noalloc_last_error "
            "abm_stepsize_set_weights "
            "abm_stepsize_get_weights abm_stepsize_get_log abm_stepsize_clear_log abm_mlp_forward "
            "abm_mlp_grad abm_mlp_train abm_mlp_last_error abm_get_adhesion_flags abm_set_adhesion_flags "
            "abm_set_cell_limit abm_batch_create abm_batch_iterate abm_batch_synchronize abm_batch_get_stream "
            "abm_batch_destroy abm_batch_last_error abm_autotune_pair_tile abm_write_cells abm_read_cells "
            "abm_write_lineage abm_read_lineage abm_io_last_error abm_set_frames abm_frames_taken "
            "abm_download_frame abm_set_switching abm_set_basal_only abm_basal_dropped").split()

CONTROLLER_REFERENCE, CONTROLLER_LEARNED, CONTROLLER_PI = 0, 1, 2
MLP_FEATURES, MLP_HIDDEN, MLP_NPARAM, MLP_LOG_COLS = 32, 64, 6337, 40


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def jkr_contact_radius(delta, Req, E, gamma):
    """jkrContactRadius(delta, Req, E, gamma).second (jkr.hpp:67-144)."""
    out = ctypes.c_double()
    rc = LIB.abm_jkr_contact_radius(delta, Req, E, gamma, ctypes.byref(out))
    if rc:
        raise RuntimeError("abm_jkr_contact_radius failed (%s)" % ERRORS.get(rc, rc))
    return out.value


def jkr_optimal_gamma(R, Rcell, E0, eqdist):
    """jkrOptimalSurfaceEnergyDensity (jkr.hpp:1369-1407): the adhesion energy density whose
    JKR force balance puts two cells at centerline distance eqdist (simulation.hpp:1354-1358)."""
    out = ctypes.c_double()
    rc = LIB.abm_jkr_optimal_gamma(R, Rcell, E0, eqdist, ctypes.byref(out))
    if rc:
        raise RuntimeError("abm_jkr_optimal_gamma failed (%s): need 2 Rcell <= eqdist < 2 R" % ERRORS.get(rc, rc))
    return out.value


def set_gamma_from_eqdist(cells, R, Rcell, E0, eqdist):
    """simulation.hpp:1354-1371: the adhesion energy density that puts two cells at eqdist
    (jkrOptimalSurfaceEnergyDensity), written into the gamma column (21) of a 3-D cells array:
    max_gamma for group-1 cells (column 20), 0 for the others.  Returns max_gamma."""
    max_gamma = jkr_optimal_gamma(R, Rcell, E0, eqdist)
    cells[:, 21] = np.where(cells[:, 20] == 1, max_gamma, 0.0)
    return max_gamma


def jkr_radius_table(R, Rcell, E0, gamma, n_mesh=100):
    """Overlap mesh LinSpaced(n, 0, 2(R - Rcell)) and radii (simulation.hpp:86-104, 1379-1382)."""
    delta = np.zeros(n_mesh)
    radius = np.zeros(n_mesh)
    rc = LIB.abm_jkr_radius_table(R, Rcell, E0, gamma, n_mesh, _dptr(delta), _dptr(radius))
    if rc:
        raise RuntimeError("abm_jkr_radius_table failed (%s)" % ERRORS.get(rc, rc))
    return delta, radius


def jkr_radius_table_variable(R, Rcell, E0, max_gamma, n_delta=100, n_gamma=100):
    """Overlap mesh LinSpaced(n_delta, 0, 2(R - Rcell)), gamma mesh LinSpaced(n_gamma, 0, max_gamma)
    and the radii on them, (n_delta, n_gamma) (simulation.hpp:120-145)."""
    delta, gamma = np.zeros(n_delta), np.zeros(n_gamma)
    radius = np.zeros((n_delta, n_gamma))
    rc = LIB.abm_jkr_radius_table_variable(R, Rcell, E0, max_gamma, n_delta, n_gamma, _dptr(delta), _dptr(gamma),
                                           _dptr(radius))
    if rc:
        raise RuntimeError("abm_jkr_radius_table_variable failed (%s)" % ERRORS.get(rc, rc))
    return delta, gamma, radius


class Simulation:
    """One device context: state, neighbor set, controller and CUDA graphs."""

    def __init__(self, gamma=100.0, n_mesh_overlap=100, jkr_table=None, **params):
        self.params, self.pdict = make_params(**params)
        if self.params.cap_cells <= 0:
            raise ValueError("cap_cells must be set")
        self._ctx = ctypes.c_void_p()
        rc = LIB.abm_create(ctypes.byref(self.params), ctypes.byref(self._ctx))
        if rc:
            msg = LIB.abm_last_error(self._ctx).decode() if self._ctx else ""
            if self._ctx:
                LIB.abm_destroy(self._ctx)
            self._ctx = None
            raise RuntimeError("abm_create failed (%s): %s" % (ERRORS.get(rc, rc), msg))
        self.ncols = None
        self.dims = 2 if self.params.dims == 2 else 3
        self.nq = 4 if self.dims == 2 else 6          # generalized coordinates per cell
        if self.params.adhesion_mode and self.dims == 3:
            if jkr_table is None:
                jkr_table = jkr_radius_table(self.params.R, self.params.Rcell, self.params.E0, gamma,
                                             n_mesh_overlap)
            self.set_jkr_table(*jkr_table)

    # -- plumbing -------------------------------------------------------------
    def _check(self, rc, what):
        if rc:
            raise RuntimeError("%s failed (%s): %s" % (what, ERRORS.get(rc, rc),
                                                       LIB.abm_last_error(self._ctx).decode()))

    def close(self):
        if self._ctx:
            LIB.abm_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        s = ctypes.c_void_p()
        self._check(LIB.abm_get_stream(self._ctx, ctypes.byref(s)), "abm_get_stream")
        return s.value

    def synchronize(self):
        self._check(LIB.abm_synchronize(self._ctx), "abm_synchronize")

    # -- state ----------------------------------------------------------------
    def set_jkr_table(self, delta, radius):
        delta = np.ascontiguousarray(delta, dtype=np.float64)
        radius = np.ascontiguousarray(radius, dtype=np.float64)
        self._check(LIB.abm_set_jkr_table(self._ctx, _dptr(delta), _dptr(radius), len(delta)),
                    "abm_set_jkr_table")

    def set_jkr_table_variable(self, delta, gamma, radius):
        """Variable-gamma JKR table (IsotropicJKRDataVariableGamma): radius (n_delta, n_gamma)."""
        delta = np.ascontiguousarray(delta, dtype=np.float64)
        gamma = np.ascontiguousarray(gamma, dtype=np.float64)
        radius = np.ascontiguousarray(radius, dtype=np.float64)
        assert radius.shape == (len(delta), len(gamma))
        self._check(LIB.abm_set_jkr_table_variable(self._ctx, _dptr(delta), len(delta), _dptr(gamma), len(gamma),
                                                   _dptr(radius)), "abm_set_jkr_table_variable")

    def set_switching(self, mode=1, rates=(0.0, 0.0, 0.0, 0.0), growth=((0.0, 0.0), (0.0, 0.0)), timescale=0.0,
                      attrs=(), max_gamma=0.0, modulate=0, visc=(0.0, 0.0, 0.0, 0.0), max_coord=1, n_start=0):
        """Phenotype switching between groups 1 and 2 (abm_set_switching): mode 1 Markov, 2 inherited
        at division; rates 2 x 2 row-major (row = current group); growth = (means, stds) per group;
        attrs = [(column, target in group 1, target in group 2), ...] for columns 17-19; gamma ramps
        to max_gamma (group 1) or 0 (group 2) over `timescale`; modulate / visc / max_coord: local
        viscosity from the group-1 share of contacts."""
        cols = (ctypes.c_int * 4)(*[int(c) for c, _, _ in attrs])
        targets = np.array([t1 for _, t1, _ in attrs] + [t2 for _, _, t2 in attrs] + [0.0], dtype=np.float64)
        rates = np.ascontiguousarray(rates, dtype=np.float64)
        gm = np.ascontiguousarray(growth[0], dtype=np.float64)
        gs = np.ascontiguousarray(growth[1], dtype=np.float64)
        visc = np.ascontiguousarray(visc, dtype=np.float64)
        self._check(LIB.abm_set_switching(self._ctx, int(mode), int(n_start), _dptr(rates), _dptr(gm), _dptr(gs),
                                          float(timescale), len(attrs), cols, _dptr(targets), float(max_gamma),
                                          int(modulate), _dptr(visc), int(max_coord)), "abm_set_switching")

    def set_basal_only(self, on=True, min_overlap=0.0):
        """Basal-only compaction after each accepted step (abm_set_basal_only)."""
        self._check(LIB.abm_set_basal_only(self._ctx, int(bool(on)), float(min_overlap)), "abm_set_basal_only")

    def basal_dropped(self):
        v = ctypes.c_longlong()
        self._check(LIB.abm_basal_dropped(self._ctx, ctypes.byref(v)), "abm_basal_dropped")
        return v.value

    def upload_cells(self, cells):
        """cells: (n, ncols) float64 array in the reference's column order."""
        a = np.asfortranarray(cells, dtype=np.float64)
        n, ncols = a.shape
        self._check(LIB.abm_upload_cells(self._ctx, _dptr(a), n, ncols, max(n, 1)), "abm_upload_cells")
        self.ncols = ncols

    def upload_cells_raw(self, ptr, n, ncols, ld):
        """Upload from a raw column-major host pointer (e.g. pinned memory)."""
        self._check(LIB.abm_upload_cells(self._ctx, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)),
                                         n, ncols, ld), "abm_upload_cells")
        self.ncols = ncols

    def download_cells(self):
        n = self.num_cells()
        out = np.zeros((n, self.ncols), dtype=np.float64, order="F")
        self._check(LIB.abm_download_cells(self._ctx, _dptr(out), max(n, 1)), "abm_download_cells")
        return out

    def download_cells_raw(self, ptr, ld):
        self._check(LIB.abm_download_cells(self._ctx, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)), ld),
                    "abm_download_cells")

    def num_cells(self):
        n = ctypes.c_int()
        self._check(LIB.abm_get_num_cells(self._ctx, ctypes.byref(n)), "abm_get_num_cells")
        return n.value

    def set_clock(self, t, dt, iteration):
        self._check(LIB.abm_set_clock(self._ctx, t, dt, iteration), "abm_set_clock")

    def clock(self):
        t, dt, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(LIB.abm_get_clock(self._ctx, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it)),
                    "abm_get_clock")
        return t.value, dt.value, it.value

    def set_parents(self, parents):
        a = np.ascontiguousarray(parents, dtype=np.int32)
        self._check(LIB.abm_set_parents(self._ctx, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(a)),
                    "abm_set_parents")

    def save_checkpoint(self, path):
        """Exact binary checkpoint (cells, neighbor set, lineage, clock, controller state)."""
        self._check(LIB.abm_save_checkpoint(self._ctx, os.fsencode(path)), "abm_save_checkpoint")

    def load_checkpoint(self, path):
        """Resume from abm_save_checkpoint's file; the context must have the saving one's
        parameters, JKR table and network weights."""
        self._check(LIB.abm_load_checkpoint(self._ctx, os.fsencode(path)), "abm_load_checkpoint")
        self.ncols = self._ckpt_cols(path)

    @staticmethod
    def _ckpt_cols(path):
        with open(path, "rb") as f:
            head = f.read(16)
        return int(np.frombuffer(head[8:16], dtype=np.int32)[1])

    def parents(self):
        n = ctypes.c_int()
        self._check(LIB.abm_get_parents(self._ctx, None, 0, ctypes.byref(n)), "abm_get_parents")
        a = np.zeros(n.value, dtype=np.int32)
        self._check(LIB.abm_get_parents(self._ctx, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n.value,
                                        ctypes.byref(n)), "abm_get_parents")
        return a

    # -- hot path ---------------------------------------------------------------
    def get_cell_neighbors(self):
        m = ctypes.c_int()
        self._check(LIB.abm_build_neighbors(self._ctx, ctypes.byref(m)), "abm_build_neighbors")
        return m.value

    def neighbors(self):
        """(m, 7) table (2-D: (m, 6)) in the reference's row order with current distances."""
        m = ctypes.c_int()
        self._check(LIB.abm_download_neighbors(self._ctx, None, 0, 0, ctypes.byref(m)), "abm_download_neighbors")
        out = np.zeros((m.value, 6 if self.dims == 2 else 7), dtype=np.float64, order="F")
        ld = max(m.value, 1)
        self._check(LIB.abm_download_neighbors(self._ctx, _dptr(out), ld, m.value, ctypes.byref(m)),
                    "abm_download_neighbors")
        return out

    def set_neighbors(self, rows):
        a = np.asfortranarray(rows, dtype=np.float64)
        self._check(LIB.abm_upload_neighbors(self._ctx, _dptr(a), a.shape[0], max(a.shape[0], 1)),
                    "abm_upload_neighbors")

    def cell_cell_forces(self):
        n = self.num_cells()
        out = np.zeros((n, self.nq), dtype=np.float64, order="F")
        self._check(LIB.abm_cell_cell_forces(self._ctx, _dptr(out)), "abm_cell_cell_forces")
        return out

    def get_velocities(self):
        n = self.num_cells()
        out = np.zeros((n, self.nq), dtype=np.float64, order="F")
        self._check(LIB.abm_get_velocities(self._ctx, _dptr(out)), "abm_get_velocities")
        return out

    def step_runge_kutta_adaptive(self, dt, attempt=0):
        """One RK attempt at dt (not accepted): (new cells, errors, scaled max error)."""
        n = self.num_cells()
        cells = np.zeros((n, self.ncols), dtype=np.float64, order="F")
        errors = np.zeros((n, self.nq), dtype=np.float64, order="F")
        e = ctypes.c_double()
        self._check(LIB.abm_rk_attempt(self._ctx, dt, attempt, _dptr(cells), _dptr(errors), ctypes.byref(e)),
                    "abm_rk_attempt")
        return cells, errors, e.value

    def grow_cells(self, dt):
        self._check(LIB.abm_grow(self._ctx, dt), "abm_grow")

    def divide_cells(self):
        """divideMaxLength + divideCells (growth.hpp:66-71, 166-426) at the current clock.

        Returns the number of mothers; the neighbor set must be rebuilt afterwards,
        as the reference loop does."""
        nd = ctypes.c_int()
        self._check(LIB.abm_divide(self._ctx, ctypes.byref(nd)), "abm_divide")
        return nd.value

    def last_division_tries(self):
        t = ctypes.c_int()
        self._check(LIB.abm_last_division_tries(self._ctx, ctypes.byref(t)), "abm_last_division_tries")
        return t.value

    def iterate(self, n_iters, n_cells_stop=0, stats=True):
        s = AbmStats()
        self._check(LIB.abm_iterate(self._ctx, n_iters, n_cells_stop, ctypes.byref(s) if stats else None),
                    "abm_iterate")
        return s.as_dict() if stats else None

    def profile_iterations(self, n_iters):
        p = AbmProfile()
        self._check(LIB.abm_profile_iterations(self._ctx, n_iters, ctypes.byref(p)), "abm_profile_iterations")
        return p.as_dict()

    def graph_info(self):
        return LIB.abm_graph_info(self._ctx).decode()

    def stats(self):
        s = AbmStats()
        self._check(LIB.abm_get_stats(self._ctx, ctypes.byref(s)), "abm_get_stats")
        return s.as_dict()

    # ---- frames of the device-resident loop (runSimulation's dt_write writes) ----
    def set_frames(self, dt_write, slots=8):
        """Mark a frame after every accepted step whose time crosses a multiple of
        dt_write (simulation.hpp:2025-2028), kept in a ring of `slots` device snapshots."""
        self._check(LIB.abm_set_frames(self._ctx, float(dt_write), int(slots)), "abm_set_frames")

    def frames_taken(self):
        k = ctypes.c_int()
        self._check(LIB.abm_frames_taken(self._ctx, ctypes.byref(k)), "abm_frames_taken")
        return k.value

    def download_frame(self, index):
        """(cells, t, iteration, lineage length) of frame `index`."""
        n, it, npar = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        t = ctypes.c_double()
        self._check(LIB.abm_download_frame(self._ctx, int(index), None, 1, ctypes.byref(n), ctypes.byref(t),
                                           ctypes.byref(it), ctypes.byref(npar)), "abm_download_frame")
        cells = np.zeros((n.value, self.ncols), dtype=np.float64, order="F")
        if n.value:
            self._check(LIB.abm_download_frame(self._ctx, int(index), cells.ctypes.data, n.value, ctypes.byref(n),
                                               ctypes.byref(t), ctypes.byref(it), ctypes.byref(npar)),
                        "abm_download_frame")
        return cells, t.value, it.value, npar.value

    def set_cell_limit(self, n_max):
        """Stop on the device once the population reaches n_max (terminate(), simulation.hpp:1600-1615)."""
        self._check(LIB.abm_set_cell_limit(self._ctx, int(n_max)), "abm_set_cell_limit")

    # ---- 2-D adhesion flags (to_adhere, 2D/include/simulation.hpp:242-258) ----
    def adhesion_flags(self):
        m = ctypes.c_int()
        self._check(LIB.abm_get_adhesion_flags(self._ctx, None, 0, ctypes.byref(m)), "abm_get_adhesion_flags")
        a = np.zeros(max(m.value, 1), dtype=np.int32)
        self._check(LIB.abm_get_adhesion_flags(self._ctx, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), m.value,
                                               ctypes.byref(m)), "abm_get_adhesion_flags")
        return a[:m.value]

    def set_adhesion_flags(self, flags):
        a = np.ascontiguousarray(flags, dtype=np.int32)
        self._check(LIB.abm_set_adhesion_flags(self._ctx, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(a)),
                    "abm_set_adhesion_flags")

    # ---- step-size network (no reference counterpart) ----
    def set_stepsize_weights(self, weights):
        w = np.ascontiguousarray(weights, dtype=np.float32).ravel()
        self._check(LIB.abm_stepsize_set_weights(self._ctx, _fptr(w), w.size), "abm_stepsize_set_weights")

    def stepsize_weights(self):
        w = np.zeros(MLP_NPARAM, dtype=np.float32)
        self._check(LIB.abm_stepsize_get_weights(self._ctx, _fptr(w), w.size), "abm_stepsize_get_weights")
        return w

    def stepsize_log(self):
        """Logged rows, oldest first: (n, 40) float32 (features, ln(dt_max/dt_first),
        ln(dt_first/dt_prev), log10 E of the first attempt, passed, error-model baseline b)."""
        cap = max(int(self.params.stepsize_log_capacity), 0)
        rows = np.zeros((max(cap, 1), MLP_LOG_COLS), dtype=np.float32)
        n = ctypes.c_int()
        self._check(LIB.abm_stepsize_get_log(self._ctx, _fptr(rows), cap, ctypes.byref(n)), "abm_stepsize_get_log")
        return rows[:n.value].copy()

    def clear_stepsize_log(self):
        self._check(LIB.abm_stepsize_clear_log(self._ctx), "abm_stepsize_clear_log")


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _mlp_check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed (%d): %s" % (what, rc, LIB.abm_mlp_last_error().decode()))


def mlp_forward(weights, X):
    """Network output ln(dt/dt_prev) for each row of X (n x 32), on the GPU."""
    w = np.ascontiguousarray(weights, dtype=np.float32).ravel()
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.zeros(X.shape[0], dtype=np.float32)
    _mlp_check(LIB.abm_mlp_forward(_fptr(w), _fptr(X), X.shape[0], _fptr(Y)), "abm_mlp_forward")
    return Y


def mlp_grad(weights, X, T):
    """(gradient of 0.5 mean (y - t)^2, loss) from the GPU backward kernels."""
    w = np.ascontiguousarray(weights, dtype=np.float32).ravel()
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    G = np.zeros(MLP_NPARAM, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    _mlp_check(LIB.abm_mlp_grad(_fptr(w), _fptr(X), _fptr(T), X.shape[0], _fptr(G), _fptr(loss)), "abm_mlp_grad")
    return G, float(loss[0])


def mlp_train(weights, X, T, epochs=200, lr=1e-3, seed=0):
    """Adam on the GPU; returns (trained weights, loss per epoch)."""
    w = np.ascontiguousarray(weights, dtype=np.float32).ravel().copy()
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    losses = np.zeros(max(epochs, 1), dtype=np.float32)
    _mlp_check(LIB.abm_mlp_train(_fptr(w), _fptr(X), _fptr(T), X.shape[0], epochs, lr, seed, _fptr(losses)),
               "abm_mlp_train")
    return w, losses[:epochs]


def _batch_check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed (%s): %s" % (what, ERRORS.get(rc, rc), LIB.abm_batch_last_error().decode()))


class Batch:
    """Independent simulations (replicate biofilms) advanced by one CUDA graph launch
    per iteration; each keeps its own clock, step size and controller."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s._ctx.value for s in self.sims])
        self._b = ctypes.c_void_p()
        _batch_check(LIB.abm_batch_create(arr, len(self.sims), ctypes.byref(self._b)), "abm_batch_create")

    def iterate(self, n_iters):
        _batch_check(LIB.abm_batch_iterate(self._b, int(n_iters)), "abm_batch_iterate")

    def synchronize(self):
        _batch_check(LIB.abm_batch_synchronize(self._b), "abm_batch_synchronize")

    @property
    def stream(self):
        s = ctypes.c_void_p()
        _batch_check(LIB.abm_batch_get_stream(self._b, ctypes.byref(s)), "abm_batch_get_stream")
        return s.value

    def close(self):
        if self._b:
            LIB.abm_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune_pair_tile(cells, launches=20, jkr_table=None, gamma=100.0, **params):
    """Time the screened pair pass on `cells` with at least 512, 1024, 2048 pairs per block
    and at most 1, 2, 4 blocks per SM; returns ((tile, blocks_per_sm), {(tile, bpsm): ms})."""
    p, d = make_params(**params)
    a = np.asfortranarray(cells, dtype=np.float64)
    if p.cap_cells <= 0:
        p.cap_cells = a.shape[0]
    if jkr_table is None and p.adhesion_mode and p.dims != 2:
        jkr_table = jkr_radius_table(p.R, p.Rcell, p.E0, gamma)
    jd = np.ascontiguousarray(jkr_table[0] if jkr_table is not None else np.zeros(2))
    jr = np.ascontiguousarray(jkr_table[1] if jkr_table is not None else np.zeros(2))
    bt, bb = ctypes.c_int(), ctypes.c_int()
    ms = np.zeros(9, dtype=np.float32)
    _batch_check(LIB.abm_autotune_pair_tile(ctypes.byref(p), _dptr(a), a.shape[0], a.shape[1], a.shape[0],
                                            _dptr(jd), _dptr(jr), len(jd), launches, ctypes.byref(bt),
                                            ctypes.byref(bb), _fptr(ms)), "abm_autotune_pair_tile")
    keys = [(t, g) for t in (512, 1024, 2048) for g in (1, 2, 4)]
    return (bt.value, bb.value), dict(zip(keys, ms.tolist()))
