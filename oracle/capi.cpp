// ORACLE — test infrastructure only (see abm3d.hpp).  A C interface over the
// 3-D restatement so the Python tests and the benchmark's CPU-baseline leg can
// drive it through ctypes.  Cell arrays are column-major n x ncols doubles,
// neighbor rows are column-major m x 7 doubles (i, j, dx, dy, dz, si, sj),
// exactly the reference's layouts.
#include <cstring>
#include <memory>
#include <string>
#include <chrono>
#include "abm3d.hpp"

using namespace oracle;

extern "C" {

struct oracle_params {
    double R, Rcell, E0, Ecell, L0, Ldiv;
    double neighbor_threshold, nz_threshold;
    int adhesion_mode, integration_mode;
    double max_stepsize, min_stepsize, max_error_allowed, min_error;
    int max_tries_update_stepsize, iter_update_stepsize, iter_update_neighbors;
    double max_rxy_noise, max_rz_noise, max_nxy_noise, max_nz_noise;
    double cell_surface_coulomb_coeff;
    int no_surface;
    double growth_mean, growth_std, daughter_length_std;
    double daughter_angle_xy_bound, daughter_angle_z_bound;
    unsigned long long rng_seed;
    int n_start_multithread;
    int n_threads;   // OpenMP threads for the reference's parallel loops (0 = default)
    int friction_mode;                // 0 NONE, 1 KINETIC cell-cell friction
    double cell_cell_coulomb_coeff;   // Coulomb cap of the friction (not positive: none)
    double M0;                        // cell mass at length L0 (velocity Verlet)
    int controller;                   // 0 the reference rule, 2 the PI controller
};

struct oracle_ctx {
    Params3 p;
    LoopState st;
    std::string err;
    std::unique_ptr<RngStream> stream;   // the reference's sequential source, when selected
};

static std::string g_last_error;

int oracle_create(const oracle_params* q, oracle_ctx** out)
{
    oracle_ctx* c = new oracle_ctx();
    Params3& p = c->p;
    p.R = q->R; p.Rcell = q->Rcell; p.E0 = q->E0; p.Ecell = q->Ecell; p.L0 = q->L0; p.Ldiv = q->Ldiv;
    p.neighbor_threshold = q->neighbor_threshold; p.nz_threshold = q->nz_threshold;
    p.adhesion_mode = q->adhesion_mode; p.integration_mode = q->integration_mode;
    p.max_stepsize = q->max_stepsize; p.min_stepsize = q->min_stepsize;
    p.max_error_allowed = q->max_error_allowed; p.min_error = q->min_error;
    p.max_tries_update_stepsize = q->max_tries_update_stepsize;
    p.iter_update_stepsize = q->iter_update_stepsize; p.iter_update_neighbors = q->iter_update_neighbors;
    p.max_rxy_noise = q->max_rxy_noise; p.max_rz_noise = q->max_rz_noise;
    p.max_nxy_noise = q->max_nxy_noise; p.max_nz_noise = q->max_nz_noise;
    p.cell_surface_coulomb_coeff = q->cell_surface_coulomb_coeff; p.no_surface = q->no_surface;
    p.growth_mean = q->growth_mean; p.growth_std = q->growth_std;
    p.daughter_length_std = q->daughter_length_std;
    p.daughter_angle_xy_bound = q->daughter_angle_xy_bound; p.daughter_angle_z_bound = q->daughter_angle_z_bound;
    p.rng_seed = q->rng_seed; p.n_start_multithread = q->n_start_multithread;
    p.friction_mode = q->friction_mode; p.cell_cell_coulomb_coeff = q->cell_cell_coulomb_coeff;
    p.M0 = q->M0;
    p.controller = q->controller;
#ifdef _OPENMP
    if (q->n_threads > 0) omp_set_num_threads(q->n_threads);
#endif
    c->st.dt = p.max_stepsize;
    *out = c;
    return 0;
}

void oracle_destroy(oracle_ctx* c) { delete c; }

const char* oracle_last_error(void) { return g_last_error.c_str(); }

int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int oracle_set_jkr_table(oracle_ctx* c, const double* delta, const double* radius, int n)
{
    c->p.jkr_overlaps.assign(delta, delta + n);
    c->p.jkr_radii.assign(radius, radius + n);
    return 0;
}

// simulation.hpp:1379-1382 mesh + simulation.hpp:86-104 radii
int oracle_jkr_table(double R, double Rcell, double E0, double gamma, int n_mesh,
                     double* delta_out, double* radius_out)
{
    std::vector<double> d = linspaced(n_mesh, 0, 2 * (R - Rcell));
    std::vector<double> r = jkr_radius_table(d, gamma, R, E0);
    for (int i = 0; i < n_mesh; ++i) { delta_out[i] = d[i]; radius_out[i] = r[i]; }
    return 0;
}

double oracle_jkr_contact_radius(double delta, double Req, double E, double gamma)
{
    return jkr_contact_radius(delta, Req, E, gamma);
}

// jkr.hpp:1311-1339, from dinit = 1.5 R with dmin = 2 Rcell as jkr.hpp:1389-1390 calls it
double oracle_jkr_equilibrium_distance(double R, double Rcell, double E0, double gamma)
{
    return jkr_equilibrium_distance(R, E0, gamma, 0.75 * 2 * R, 2 * Rcell, 1e-8, 1e-8, 1000);
}

// jkr.hpp:1369-1407 as simulation.hpp:1355-1358 calls it
double oracle_jkr_optimal_gamma(double R, double Rcell, double E0, double eqdist)
{
    return jkr_optimal_gamma(R, Rcell, E0, eqdist);
}

int oracle_set_cells(oracle_ctx* c, const double* colmajor, int n, int ncols, int ld)
{
    Cells cells(n, ncols);
    for (int j = 0; j < ncols; ++j)
        for (int i = 0; i < n; ++i) cells(i, j) = colmajor[(size_t)j * ld + i];
    c->st.cells = cells;
    c->st.nb = Neighbors();
    return 0;
}

int oracle_get_num_cells(oracle_ctx* c) { return c->st.cells.n; }

int oracle_get_cells(oracle_ctx* c, double* colmajor, int ld)
{
    const Cells& cells = c->st.cells;
    for (int j = 0; j < cells.ncols; ++j)
        for (int i = 0; i < cells.n; ++i) colmajor[(size_t)j * ld + i] = cells(i, j);
    return 0;
}

int oracle_set_parents(oracle_ctx* c, const int* parents, int n)
{
    c->st.parents.assign(parents, parents + n);
    return 0;
}

int oracle_get_parents(oracle_ctx* c, int* out, int cap)
{
    int n = (int)c->st.parents.size();
    for (int i = 0; i < n && i < cap; ++i) out[i] = c->st.parents[i];
    return n;
}

void oracle_set_clock(oracle_ctx* c, double t, double dt, int iter)
{
    c->st.t = t; c->st.dt = dt; c->st.iter = iter;
}

void oracle_get_clock(oracle_ctx* c, double* t, double* dt, int* iter)
{
    *t = c->st.t; *dt = c->st.dt; *iter = c->st.iter;
}

// mechanics.hpp:520-593
int oracle_build_neighbors(oracle_ctx* c)
{
    c->st.nb = build_neighbors(c->st.cells, c->p);
    return c->st.nb.size();
}

// the "optimized CPU" procedures (cell-list neighbor build, OpenMP over the pairs), for
// the context figure beside the reference-faithful CPU run; off by default
void oracle_set_cpu_optimized(oracle_ctx* c, int on) { c->p.cpu_optimized = on ? 1 : 0; }

// on = 1: every random draw comes from one mt19937 seeded with `seed`, in the reference's
// order (the semantics check of its random source); on = 0: the Philox counter policy
void oracle_set_rng_stream(oracle_ctx* c, int on, unsigned seed)
{
    c->stream.reset(on ? new RngStream(seed) : nullptr);
    c->p.stream = c->stream.get();
}

// uniforms drawn from the stream so far (0 without one)
long long oracle_rng_stream_draws(oracle_ctx* c) { return c->stream ? c->stream->draws : 0; }

// the first k uniforms of a fresh stream seeded with `seed`
void oracle_rng_stream_uniforms(unsigned seed, int k, double* out)
{
    RngStream r(seed);
    for (int i = 0; i < k; ++i) out[i] = r.uniform01();
}

int oracle_num_neighbors(oracle_ctx* c) { return c->st.nb.size(); }

// column-major m x 7 rows (ld = m)
int oracle_get_neighbors(oracle_ctx* c, double* out, int ld)
{
    const Neighbors& nb = c->st.nb;
    for (int k = 0; k < nb.size(); ++k)
    {
        out[k] = nb.i[k]; out[ld + k] = nb.j[k];
        out[2 * ld + k] = nb.dx[k]; out[3 * ld + k] = nb.dy[k]; out[4 * ld + k] = nb.dz[k];
        out[5 * ld + k] = nb.si[k]; out[6 * ld + k] = nb.sj[k];
    }
    return nb.size();
}

int oracle_set_neighbors(oracle_ctx* c, const double* rows, int m, int ld)
{
    Neighbors nb;
    for (int k = 0; k < m; ++k)
    {
        nb.i.push_back((int)rows[k]); nb.j.push_back((int)rows[ld + k]);
        nb.dx.push_back(rows[2 * ld + k]); nb.dy.push_back(rows[3 * ld + k]); nb.dz.push_back(rows[4 * ld + k]);
        nb.si.push_back(rows[5 * ld + k]); nb.sj.push_back(rows[6 * ld + k]);
    }
    c->st.nb = nb;
    return 0;
}

// mechanics.hpp:604-648
int oracle_update_neighbor_distances(oracle_ctx* c)
{
    update_neighbor_distances(c->st.cells, c->st.nb);
    return 0;
}

// distances.hpp:206-357 ; out = (dx, dy, dz, s, t)
void oracle_dist_between_cells(const double* r1, const double* n1, double h1,
                               const double* r2, const double* n2, double h2, double* out)
{
    DistResult d = dist_between_cells(v3(r1[0], r1[1], r1[2]), v3(n1[0], n1[1], n1[2]), h1,
                                      v3(r2[0], r2[1], r2[2]), v3(n2[0], n2[1], n2[2]), h2);
    out[0] = d.d.x; out[1] = d.d.y; out[2] = d.d.z; out[3] = d.s; out[4] = d.t;
}

// distances.hpp:92-105
double oracle_nearest_body_coord(const double* r, const double* n, double h, const double* q)
{
    return nearest_body_coord(v3(r[0], r[1], r[2]), v3(n[0], n[1], n[2]), h, v3(q[0], q[1], q[2]));
}

// mechanics.hpp:1209-1659: dE/dq (n x 6 column-major) from the current table
int oracle_cell_cell_forces(oracle_ctx* c, double* out)
{
    try
    {
        Arr6 f = cell_cell_forces(c->st.cells, c->st.nb, c->p);
        add_friction(f, c->st.cells, c->st.nb, c->p);   // mechanics.hpp:1339-1346
        std::memcpy(out, f.data(), f.size() * sizeof(double));
    }
    catch (const std::exception& e) { g_last_error = e.what(); return -1; }
    return 0;
}

// mechanics.hpp:1702-1769 with assume_2d from the current cells
int oracle_conservative_forces(oracle_ctx* c, double* out)
{
    const Cells& cells = c->st.cells;
    std::vector<int> a2(cells.n);
    for (int i = 0; i < cells.n; ++i) a2[i] = cells(i, C_NZ) < c->p.nz_threshold;
    try
    {
        Arr6 f = get_conservative_forces(cells, c->st.nb, c->p, a2, false);
        std::memcpy(out, f.data(), f.size() * sizeof(double));
    }
    catch (const std::exception& e) { g_last_error = e.what(); return -1; }
    return 0;
}

// mechanics.hpp:2011-2347 without noise
int oracle_get_velocities(oracle_ctx* c, double* out)
{
    const Cells& cells = c->st.cells;
    std::vector<int> a2(cells.n);
    for (int i = 0; i < cells.n; ++i) a2[i] = cells(i, C_NZ) < c->p.nz_threshold;
    Arr6 noise((size_t)cells.n * 6, 0.0);
    try
    {
        Arr6 v = get_velocities(cells, c->st.nb, c->p, a2, noise, false);
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    }
    catch (const std::exception& e) { g_last_error = e.what(); return -1; }
    return 0;
}

// mechanics.hpp:2406-2612 for one attempt at dt (does not modify the state).
// cells_out: n x ncols column-major (ld = n); errors_out: n x 6.
int oracle_rk_attempt(oracle_ctx* c, double dt, int iter, int attempt, double* cells_out,
                      double* errors_out, double* max_err)
{
    try
    {
        Tableau tab = make_tableau(c->p.integration_mode);
        Arr6 errors;
        Cells cn = step_rk_adaptive(tab, c->st.cells, c->st.nb, dt, c->p, iter, attempt, errors, true);
        if (cells_out) std::memcpy(cells_out, cn.a.data(), cn.a.size() * sizeof(double));
        if (errors_out) std::memcpy(errors_out, errors.data(), errors.size() * sizeof(double));
        if (max_err) *max_err = max_scaled_error(c->st.cells, errors, c->p.max_error_allowed, c->p.min_error);
    }
    catch (const std::exception& e) { g_last_error = e.what(); return -1; }
    return 0;
}

// simulation.hpp:1277 initial neighbor build and dt = max_stepsize
int oracle_loop_init(oracle_ctx* c)
{
    loop_init(c->st, c->p);
    return c->st.nb.size();
}

// simulation.hpp:1617-1864 for n_iters iterations (stops early once the cell
// count reaches n_cells when n_cells > 0).  fast_cc = 1 evaluates the
// stage-invariant pair forces once per attempt (same arithmetic).
int oracle_iterate(oracle_ctx* c, int n_iters, int n_cells, int fast_cc)
{
    try
    {
        for (int k = 0; k < n_iters; ++k)
        {
            if (n_cells > 0 && c->st.cells.n >= n_cells) break;
            loop_iteration(c->st, c->p, fast_cc != 0);
        }
    }
    catch (const std::exception& e)
    {
        g_last_error = e.what();
        return -1;
    }
    return 0;
}

void oracle_get_stats(oracle_ctx* c, long long* attempts, long long* rebuilds,
                      long long* divisions, double* last_max_error)
{
    *attempts = c->st.attempts; *rebuilds = c->st.rebuilds;
    *divisions = c->st.divisions; *last_max_error = c->st.last_max_error;
}

// iterations whose first attempt failed the error test
long long oracle_rejected(oracle_ctx* c) { return c->st.rejected; }

// growth.hpp:51-57
int oracle_grow(oracle_ctx* c, double dt)
{
    grow_cells(c->st.cells, dt, c->p.R);
    return 0;
}

// growth.hpp:66-71 + 166-426 at iteration `iter`; returns the number of tries
int oracle_divide(oracle_ctx* c, double t, int iter)
{
    std::vector<int> to_divide(c->st.cells.n);
    for (int i = 0; i < c->st.cells.n; ++i) to_divide[i] = c->st.cells(i, C_L) > c->p.Ldiv;
    int ntries = 0;
    c->st.cells = divide_cells(c->st.cells, c->st.parents, t, c->p, to_divide, iter, &ntries);
    return ntries;
}

// growth.hpp:82-117
double oracle_min_dist_to_cell(oracle_ctx* c, int i)
{
    return min_dist_to_cell(c->st.cells, i);
}

// Philox policy check: one uniform
double oracle_rng_uniform(unsigned long long seed, unsigned purpose, unsigned a, unsigned b,
                          unsigned cc, unsigned d)
{
    return rng_uniform(seed, purpose, a, b, cc, d);
}

// deterministic log / sincos used by the division draws
double oracle_det_log(double x) { return det_log(x); }
void oracle_det_sincos(double x, double* s, double* c) { det_sincos(x, *s, *c); }

// integrals.hpp:400-463
void oracle_area_integrals(double rz, double nz, double R, double half_l, double* out)
{
    double ss = sstar(rz, nz, R);
    area_integrals(rz, nz, R, half_l, ss, out[0], out[1], out[2]);
}

// the auxiliary integrals of integrals.hpp (integral1, integral2, integral4-6), for the
// reference's own quadrature tests (test/src/testIntegrals.cpp)
double oracle_integral1(double rz, double nz, double R, double half_l, double gamma, double ss)
{
    return integral1(rz, nz, R, half_l, gamma, ss);
}
double oracle_integral2(double rz, double nz, double R, double half_l, double gamma, double ss)
{
    return integral2(rz, nz, R, half_l, gamma, ss);
}
double oracle_integral4(double nz, double half_l, double ss) { return integral4(nz, half_l, ss); }
double oracle_integral5(double nz, double half_l, double ss) { return integral5(nz, half_l, ss); }
double oracle_integral6(double nz, double half_l, double ss) { return integral6(nz, half_l, ss); }

// cellSurfaceRepulsionForces (kind 0, mechanics.hpp:673-780) or cellSurfaceAdhesionForces
// (kind 1, mechanics.hpp:800-910) of one cell with center height rz, orientation
// (nx, 0, nz), half-length half_l and adhesion energy density sigma0, treated as
// horizontal when nz < nz_threshold; the six generalized forces go to out6, in the
// include_constraint form when `constraint` is set (the velocity-Verlet path).  This is the
// single-cell form the reference's own tests call (testCellSurfaceRepulsionForces.cpp,
// testCellSurfaceAdhesionForces.cpp), with ss = (R - rz) / nz.
int oracle_surface_forces(int kind, double rz, double nx, double nz, double half_l, double sigma0,
                          double R, double E0, double nz_threshold, int constraint, double* out6)
{
    if (kind != 0 && kind != 1) return 1;
    Cells cells(1, NCOLS_REQUIRED_3D);
    cells(0, C_RZ) = rz; cells(0, C_NX) = nx; cells(0, C_NZ) = nz;
    cells(0, C_L) = 2 * half_l; cells(0, C_HALF_L) = half_l; cells(0, C_SIGMA0) = sigma0;
    std::vector<double> ss(1, sstar(rz, nz, R));
    std::vector<int> assume_2d(1, nz < nz_threshold);
    Arr6 f = kind == 0 ? cell_surface_repulsion_forces(cells, ss, R, E0, assume_2d, false, constraint != 0)
                       : cell_surface_adhesion_forces(cells, ss, R, assume_2d, false, constraint != 0);
    for (int k = 0; k < 6; ++k) out6[k] = f[k];
    return 0;
}

// simulation.hpp:1379-1395 with variable gamma: overlap mesh LinSpaced(nd, 0, 2 (R - Rcell)),
// gamma mesh LinSpaced(ng, 0, max_gamma), radii nd x ng overlap-major
int oracle_jkr_table2(double R, double Rcell, double E0, double max_gamma, int nd, int ng,
                      double* delta_out, double* gamma_out, double* radius_out)
{
    std::vector<double> d = linspaced(nd, 0, 2 * (R - Rcell)), g = linspaced(ng, 0, max_gamma);
    std::vector<double> r = jkr_radius_table2(d, g, R, E0);
    for (int i = 0; i < nd; ++i) delta_out[i] = d[i];
    for (int j = 0; j < ng; ++j) gamma_out[j] = g[j];
    for (size_t k = 0; k < r.size(); ++k) radius_out[k] = r[k];
    return 0;
}

// install a variable-gamma table (IsotropicJKRDataVariableGamma, mechanics.hpp:159-199)
int oracle_set_jkr_table2(oracle_ctx* c, const double* delta, int nd, const double* gamma, int ng,
                          const double* radius)
{
    c->p.jkr_overlaps.assign(delta, delta + nd);
    c->p.jkr_gammas.assign(gamma, gamma + ng);
    c->p.jkr_radii2.assign(radius, radius + (size_t)nd * ng);
    return 0;
}

// phenotype switching (the f4 row): mode 0 NONE, 1 MARKOV, 2 INHERIT; rates 2 x 2 row-major
// (row = current group); growth mean / std per group; n_attr switched attributes at columns
// attr_col with targets attr_targets (2 x n_attr row-major, group 1 then group 2);
// max_gamma for the gamma ramp; viscosity limits 2 x 2 (min, max per group) when modulate.
int oracle_set_switching(oracle_ctx* c, int mode, int n_start, const double* rates, const double* growth_mean,
                         const double* growth_std, double timescale, int n_attr, const int* attr_col,
                         const double* attr_targets, double max_gamma, int modulate, const double* visc_lims,
                         int max_coord)
{
    Params3& p = c->p;
    if (mode < 0 || mode > 2 || n_attr < 0 || n_attr > 4 || max_coord < 1) return 1;
    p.switch_mode = mode; p.n_cells_start_switch = n_start;
    for (int k = 0; k < 4; ++k) p.switch_rates[k] = rates[k];
    for (int g = 0; g < 2; ++g) { p.group_growth_mean[g] = growth_mean[g]; p.group_growth_std[g] = growth_std[g]; }
    p.switch_timescale = timescale;
    p.n_attributes = n_attr;
    for (int k = 0; k < n_attr; ++k)
    {
        p.attr_col[k] = attr_col[k];
        p.attr_target[0][k] = attr_targets[k];
        p.attr_target[1][k] = attr_targets[n_attr + k];
    }
    p.max_gamma = max_gamma;
    p.modulate_local_viscosity = modulate;
    for (int k = 0; k < 4; ++k) p.viscosity_lims[k] = visc_lims ? visc_lims[k] : 0.0;
    p.max_coordination_number = max_coord;
    return 0;
}

int oracle_set_basal(oracle_ctx* c, int basal_only, double min_overlap)
{
    c->p.basal_only = basal_only; c->p.basal_min_overlap = min_overlap;
    return 0;
}

// the pieces on their own, on the context's cells
int oracle_switch_markov(oracle_ctx* c, double dt, int iter) { return switch_groups_markov(c->st.cells, c->p, dt, iter); }

int oracle_switch_inherit(oracle_ctx* c, const int* pairs, int n_pairs, int iter)
{
    std::vector<std::pair<int, int> > v;
    for (int q = 0; q < n_pairs; ++q) v.push_back(std::make_pair(pairs[2 * q], pairs[2 * q + 1]));
    return switch_groups_inherit(c->st.cells, v, c->p, iter);
}

// simulation.hpp:1872-2022 on the context's cells and neighbor rows
int oracle_switch_ramps(oracle_ctx* c, double dt)
{
    ramp_attributes(c->st.cells, c->p, dt);
    if (c->p.adhesion_mode != 0)
    {
        ramp_gamma(c->st.cells, c->p, dt);
        if (c->p.modulate_local_viscosity) modulate_viscosity(c->st.cells, c->st.nb, c->p);
    }
    return 0;
}

int oracle_basal_compact(oracle_ctx* c) { return basal_compact(c->st.cells, c->p); }

}   // extern "C"
