// ORACLE — test infrastructure only (see abm2d.hpp).  A C interface over the
// 2-D restatement for the Python tests.  Cell arrays are column-major n x ncols
// doubles in the 2-D reference layout (ABM-2d/ABM-2d-cpp/include/indices.hpp),
// neighbor rows are column-major m x 6 doubles (i, j, dx, dy, si, sj).
#include <cstring>
#include <memory>
#include <string>
#include "abm2d.hpp"

using namespace oracle;

extern "C" {

struct oracle2d_params {
    double R, Rcell, E0, Ecell, sigma0, Ldiv, neighbor_threshold;
    int adhesion_mode;
    double adhesion_strength, adhesion_mindist;
    int integration_mode;
    double max_stepsize, min_stepsize, max_error_allowed, min_error;
    int max_tries_update_stepsize, iter_update_stepsize, iter_update_neighbors;
    double max_noise, growth_mean, growth_std, daughter_length_std, daughter_angle_bound;
    unsigned long long rng_seed;
    int use_pf;
    double pf[3];
};

struct oracle2d_ctx {
    Params2 p;
    LoopState2 st;
    std::unique_ptr<RngStream> stream;   // the reference's sequential source, when selected
};

// on = 1: every random draw comes from one mt19937 seeded with `seed`, in the 2-D
// reference's order; on = 0: the Philox counter policy
void oracle2d_set_rng_stream(oracle2d_ctx* c, int on, unsigned seed)
{
    c->stream.reset(on ? new RngStream(seed) : nullptr);
    c->p.stream = c->stream.get();
}

long long oracle2d_rng_stream_draws(oracle2d_ctx* c) { return c->stream ? c->stream->draws : 0; }

int oracle2d_create(const oracle2d_params* q, oracle2d_ctx** out)
{
    oracle2d_ctx* c = new oracle2d_ctx();
    Params2& p = c->p;
    p.R = q->R; p.Rcell = q->Rcell; p.E0 = q->E0; p.Ecell = q->Ecell; p.sigma0 = q->sigma0;
    p.Ldiv = q->Ldiv; p.neighbor_threshold = q->neighbor_threshold;
    p.adhesion_mode = q->adhesion_mode; p.adhesion_strength = q->adhesion_strength;
    p.adhesion_mindist = q->adhesion_mindist; p.integration_mode = q->integration_mode;
    p.max_stepsize = q->max_stepsize; p.min_stepsize = q->min_stepsize;
    p.max_error_allowed = q->max_error_allowed; p.min_error = q->min_error;
    p.max_tries_update_stepsize = q->max_tries_update_stepsize;
    p.iter_update_stepsize = q->iter_update_stepsize; p.iter_update_neighbors = q->iter_update_neighbors;
    p.max_noise = q->max_noise; p.growth_mean = q->growth_mean; p.growth_std = q->growth_std;
    p.daughter_length_std = q->daughter_length_std; p.daughter_angle_bound = q->daughter_angle_bound;
    p.rng_seed = q->rng_seed;
    p.use_pf = q->use_pf;
    for (int k = 0; k < 3; ++k) p.pf[k] = q->pf[k];
    c->st.dt = p.max_stepsize;
    *out = c;
    return 0;
}

void oracle2d_destroy(oracle2d_ctx* c) { delete c; }

int oracle2d_set_cells(oracle2d_ctx* c, const double* cm, int n, int ncols, int ld)
{
    if (ncols < NCOLS_2D) return -1;
    Cells cells(n, ncols);
    for (int k = 0; k < ncols; ++k)
        for (int i = 0; i < n; ++i) cells(i, k) = cm[(size_t)k * ld + i];
    c->st.cells = cells;
    return 0;
}

int oracle2d_get_num_cells(oracle2d_ctx* c) { return c->st.cells.n; }

int oracle2d_get_cells(oracle2d_ctx* c, double* cm, int ld)
{
    const Cells& cells = c->st.cells;
    for (int k = 0; k < cells.ncols; ++k)
        for (int i = 0; i < cells.n; ++i) cm[(size_t)k * ld + i] = cells(i, k);
    return 0;
}

int oracle2d_set_parents(oracle2d_ctx* c, const int* parents, int n)
{
    c->st.parents.assign(parents, parents + n);
    return 0;
}

int oracle2d_get_parents(oracle2d_ctx* c, int* out, int cap)
{
    const int n = (int)c->st.parents.size();
    for (int k = 0; k < n && k < cap; ++k) out[k] = c->st.parents[k];
    return n;
}

void oracle2d_set_clock(oracle2d_ctx* c, double t, double dt, int iter)
{
    c->st.t = t; c->st.dt = dt; c->st.iter = iter;
}

void oracle2d_get_clock(oracle2d_ctx* c, double* t, double* dt, int* iter)
{
    *t = c->st.t; *dt = c->st.dt; *iter = c->st.iter;
}

int oracle2d_build_neighbors(oracle2d_ctx* c)
{
    c->st.nb = get_cell_neighbors_2d(c->st.cells, c->p);
    return c->st.nb.size();
}

int oracle2d_num_neighbors(oracle2d_ctx* c) { return c->st.nb.size(); }

// rows (i, j, dx, dy, si, sj) column-major with leading dimension ld; adhere[m]
int oracle2d_get_neighbors(oracle2d_ctx* c, double* out, int ld, int* adhere)
{
    const Neighbors2& nb = c->st.nb;
    for (int k = 0; k < nb.size(); ++k)
    {
        out[k] = nb.i[k]; out[(size_t)ld + k] = nb.j[k];
        out[2 * (size_t)ld + k] = nb.dx[k]; out[3 * (size_t)ld + k] = nb.dy[k];
        out[4 * (size_t)ld + k] = nb.si[k]; out[5 * (size_t)ld + k] = nb.sj[k];
        if (adhere) adhere[k] = nb.adhere[k];
    }
    return nb.size();
}

static void copy4(const Arr4& a, int n, double* out)
{
    for (int k = 0; k < 4; ++k)
        for (int i = 0; i < n; ++i) out[(size_t)k * n + i] = a[(size_t)k * n + i];
}

// dE/dq of the cell-cell forces (repulsion + adhesion), n x 4
int oracle2d_cell_cell_forces(oracle2d_ctx* c, double* out)
{
    const int n = c->st.cells.n;
    Arr4 rep = repulsive_forces_2d(c->st.cells, c->st.nb, c->p);
    Arr4 adh = adhesive_forces_2d(c->st.cells, c->st.nb, c->p);
    for (size_t k = 0; k < rep.size(); ++k) rep[k] += adh[k];
    copy4(rep, n, out);
    return 0;
}

int oracle2d_get_velocities(oracle2d_ctx* c, double* out)
{
    const int n = c->st.cells.n;
    Arr4 noise((size_t)n * 4, 0.0);
    copy4(get_velocities_2d(c->st.cells, c->st.nb, c->p, noise), n, out);
    return 0;
}

int oracle2d_rk_attempt(oracle2d_ctx* c, double dt, int iter, int attempt, double* cells_out,
                        double* errors_out, double* max_error)
{
    const Tableau tab = make_tableau(c->p.integration_mode);
    Arr4 errors;
    Cells cn = step_rk_2d(tab, c->st.cells, c->st.nb, dt, c->p, iter, attempt, errors);
    const int n = cn.n;
    for (int k = 0; k < cn.ncols; ++k)
        for (int i = 0; i < n; ++i) cells_out[(size_t)k * n + i] = cn(i, k);
    copy4(errors, n, errors_out);
    *max_error = max_scaled_error_2d(c->st.cells, errors, c->p.max_error_allowed, c->p.min_error);
    return 0;
}

int oracle2d_loop_init(oracle2d_ctx* c)
{
    loop_init_2d(c->st, c->p);
    return c->st.nb.size();
}

int oracle2d_iterate(oracle2d_ctx* c, int n_iters, int n_cells)
{
    for (int k = 0; k < n_iters; ++k)
    {
        if (n_cells > 0 && c->st.cells.n >= n_cells) return k;
        loop_iteration_2d(c->st, c->p);
    }
    return n_iters;
}

void oracle2d_get_stats(oracle2d_ctx* c, long long* attempts, long long* rebuilds, long long* divisions,
                        double* last_max_error)
{
    *attempts = c->st.attempts; *rebuilds = c->st.rebuilds; *divisions = c->st.divisions;
    *last_max_error = c->st.last_max_error;
}

int oracle2d_divide(oracle2d_ctx* c, double t, int iter, int* ntries)
{
    std::vector<int> to_divide(c->st.cells.n);
    int nd = 0;
    for (int i = 0; i < c->st.cells.n; ++i) { to_divide[i] = c->st.cells(i, D_L) > c->p.Ldiv; nd += to_divide[i]; }
    c->st.cells = divide_cells_2d(c->st.cells, c->st.parents, t, c->p, to_divide, iter, ntries);
    return nd;
}

// forcesJKRLagrange (2D/include/adhesion.hpp:403-448, include_constraint = true)
// for one pair: out is 2 x 4 row-major (cell 1 then cell 2), strength 1
void oracle2d_jkr_lagrange_pair(const double* n1, const double* n2, const double* d12, double R, double s,
                                double t, double dmin, double* out)
{
    Cells cells(2, NCOLS_2D);
    cells(0, D_NX) = n1[0]; cells(0, D_NY) = n1[1]; cells(1, D_NX) = n2[0]; cells(1, D_NY) = n2[1];
    cells(0, D_L) = cells(1, D_L) = 1.0;
    Neighbors2 nb;
    nb.i = {0}; nb.j = {1}; nb.dx = {d12[0]}; nb.dy = {d12[1]}; nb.si = {s}; nb.sj = {t}; nb.adhere = {1};
    Params2 p;
    p.R = R; p.adhesion_mode = 1; p.adhesion_strength = 1.0; p.adhesion_mindist = dmin;
    Arr4 f = adhesive_forces_2d(cells, nb, p);
    for (int r = 0; r < 2; ++r)
        for (int k = 0; k < 4; ++k) out[r * 4 + k] = f[(size_t)k * 2 + r];
}

int oracle2d_grow(oracle2d_ctx* c, double dt)
{
    grow_cells_2d(c->st.cells, dt, c->p.R);
    return 0;
}

}   // extern "C"
