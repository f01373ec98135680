// C ABI of the B200 mechanics step (declared in include/abm_capi.h).
//
// A context owns the device state (cell records, CSR neighbor set, cell-list
// buffers, controller state), one CUDA stream and two CUDA graphs: one loop
// iteration (pair force -> trial attempt -> retries -> final attempt with
// growth) and one neighbor rebuild (bbox -> counting sort -> pair build ->
// CSR).  All sizes that change during a run (cell count, pair count, bin
// count) live in device memory, so the graphs are captured once and replayed.
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <functional>
#include "abm_kernels.cuh"
#include "../../include/abm_capi.h"

using namespace abm;

struct abm_ctx {
    abm_params p;
    std::string err;
    int dev = 0, num_sms = 148;
    cudaStream_t st = nullptr;
    int cap = 0, cap_bins = 0, cap_nbr = 0;
    int ncols = 0, has_gamma = 0;
    int n_host = 0;
    bool cells_loaded = false, nbrs_valid = false;
    int host_iter = 0;
    // device state
    Geom* geom = nullptr; Vel* vel = nullptr; Phys* phys = nullptr; Gen6* fcc = nullptr;
    Geom* geom_c = nullptr; Vel* vel_c = nullptr; Gen6* gen_tmp = nullptr; Gen6* k0buf = nullptr;
    Ctrl* ctrl = nullptr; Grid* grid = nullptr;
    unsigned long long* bbox_acc = nullptr; unsigned int* bbox_counter = nullptr;
    int *bin_count = nullptr, *bin_start = nullptr, *key = nullptr, *slot = nullptr, *sorted_cell = nullptr;
    Geom* sorted_geom = nullptr;
    int *scratch = nullptr, *nbr_count = nullptr, *row_ptr = nullptr, *col = nullptr;
    int *lower_end = nullptr, *rev = nullptr;
    int4* pairs = nullptr;                                           // screened pair pass
    int *pair_start = nullptr, *surv = nullptr;
    double4* jbuf = nullptr;
    int* scan_sums = nullptr;
    double *jkr_delta = nullptr, *jkr_radius = nullptr;
    int jkr_n = 0;
    double *jkr_gam = nullptr, *jkr_rad2 = nullptr;    // variable-gamma table (jkr_n x fp.jkr_ng)
    double* staging = nullptr;   // cap x (ncols max 32) doubles
    // division
    DivideParams dp;
    bool div_enabled = false;
    int cap_parents = 0;
    int *div_flags = nullptr, *div_rank = nullptr, *mothers = nullptr, *div_check = nullptr, *div_sat = nullptr;
    int *div_ok = nullptr, *parents_dev = nullptr;
    Geom *d1 = nullptr, *d2 = nullptr;
    double *dlen = nullptr, *dgrowth = nullptr;
    // step-size network and its features
    float* mlp_w = nullptr;          // ABM_MLP_NPARAM FP32 master weights
    float* log_buf = nullptr;        // stepsize_log_capacity rows of MLP_LOG_COLS floats
    double4* stat_part = nullptr;    // per-block feature partials of the final attempt
    int *order = nullptr, *order_flag = nullptr, *order_pos = nullptr;   // attempt order (3-D)
    // frames: a ring of frame_slots snapshots of the cells (abm_set_frames)
    int frame_slots = 0;
    Geom* snap_geom = nullptr;
    Vel* snap_vel = nullptr;
    Phys* snap_phys = nullptr;
    FrameInfo* frame_info = nullptr;
    bool mlp_loaded = false;
    // cell-cell kinetic friction: the coefficient of each cell (column eta_col), the per-entry
    // planar-contact records, the candidate list and the stage states of the trial passes
    double* feta = nullptr;
    double4* fbuf = nullptr;
    int *fmask = nullptr, *fr_list = nullptr;
    double2* ystage = nullptr;
    double* snap_feta = nullptr;
    int eta_col = 21;
    // velocity Verlet (integration mode 0): JKR parts of the pair shares, half-step
    // angular velocities, the cell density
    bool verlet = false;
    double4 *pbuf = nullptr, *whalf = nullptr;
    double rho = 0.0;
    // phenotype switching, ramps, local viscosity, basal-only compaction (abm_switch.cu)
    SwitchParams sw;
    bool post_on = false;            // the post-step kernels run after each accepted step
    Phys* phys_c = nullptr;          // compaction scratch (geom_c / vel_c hold the rest)
    int *keep = nullptr, *keep_rank = nullptr;
    // 2-D model
    int dims = 3;
    unsigned char* adhere = nullptr;  // to_adhere per CSR entry
    // parameters
    ForceParams fp; StepParams sp; BuildParams bp;
    // graphs
    cudaGraphExec_t g_iter = nullptr, g_rebuild = nullptr;
    cudaGraphExec_t g_iter_k = nullptr;   // iter_k iterations in one graph (long loops)
    int iter_k = 1;
    bool graph_fallback = false;     // conditional nodes could not be built
    std::string graph_note;
};

static const int STAGING_COLS = 32;

#define CK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { \
    if (c) c->err = std::string(#call) + ": " + cudaGetErrorString(e_); return ABM_ERR_CUDA; } } while (0)

static int fail(abm_ctx* c, int code, const std::string& msg) { if (c) c->err = msg; return code; }

// --------------------------------------------------------------------------
// JKR contact radius: the largest real root of
//   p(a) = a^4 - 2 Req delta a^2 - (4 pi gamma Req^2 / E) a + delta^2 Req^2
// (jkr.hpp:81-84).  Newton's method started at the Cauchy bound converges
// monotonically from above to the largest real root, because by Gauss-Lucas
// the roots of p' and p'' also lie below that bound.
// --------------------------------------------------------------------------
static double jkr_radius_host(double delta, double Req, double E, double gamma)
{
    // gamma = 0: p(a) = (a^2 - Req delta)^2, a double root that Newton approaches only
    // linearly; its value is the Hertz radius
    if (gamma == 0) return std::sqrt(Req * delta);
    typedef long double LD;
    const LD pi = 3.141592653589793238462643383279502884L;
    LD c2 = -2.0L * Req * delta, c1 = -4.0L * pi * gamma * (LD)Req * Req / E, c0 = (LD)delta * delta * Req * Req;
    LD x = 1.0L + std::max(std::fabs(c2), std::max(std::fabs(c1), std::fabs(c0)));
    for (int it = 0; it < 500; ++it)
    {
        LD p = ((x * x + c2) * x + c1) * x + c0;
        LD dp = (4.0L * x * x + 2.0L * c2) * x + c1;
        if (dp <= 0) break;
        LD xn = x - p / dp;
        if (!(xn < x)) break;
        x = xn;
    }
    return (double)x;
}

extern "C" {

int abm_jkr_contact_radius(double delta, double Req, double E, double gamma, double* radius)
{
    if (!radius || Req <= 0 || E <= 0 || gamma < 0 || delta < 0) return ABM_ERR_ARG;
    *radius = jkr_radius_host(delta, Req, E, gamma);
    return ABM_OK;
}

int abm_jkr_radius_table(double R, double Rcell, double E0, double gamma, int n_mesh,
                         double* delta_out, double* radius_out)
{
    if (n_mesh < 2 || !delta_out || !radius_out) return ABM_ERR_ARG;
    // Eigen LinSpaced(n, 0, 2 (R - Rcell)): low + i * step, last entry exactly high
    const double high = 2 * (R - Rcell), step = (high - 0.0) / double(n_mesh - 1);
    for (int i = 0; i < n_mesh; ++i)
    {
        delta_out[i] = (i == n_mesh - 1) ? high : 0.0 + double(i) * step;
        radius_out[i] = jkr_radius_host(delta_out[i], R / 2, E0, gamma);
    }
    return ABM_OK;
}

int abm_jkr_radius_table_variable(double R, double Rcell, double E0, double max_gamma, int n_delta, int n_gamma,
                                  double* delta_out, double* gamma_out, double* radius_out)
{
    if (n_delta < 2 || n_gamma < 2 || !(max_gamma > 0) || !delta_out || !gamma_out || !radius_out)
        return ABM_ERR_ARG;
    const double high = 2 * (R - Rcell), step = high / double(n_delta - 1), gstep = max_gamma / double(n_gamma - 1);
    for (int i = 0; i < n_delta; ++i) delta_out[i] = (i == n_delta - 1) ? high : double(i) * step;
    for (int j = 0; j < n_gamma; ++j) gamma_out[j] = (j == n_gamma - 1) ? max_gamma : double(j) * gstep;
    for (int i = 0; i < n_delta; ++i)
        for (int j = 0; j < n_gamma; ++j)
            radius_out[(size_t)i * n_gamma + j] = jkr_radius_host(delta_out[i], R / 2, E0, gamma_out[j]);
    return ABM_OK;
}

// jkrOptimalSurfaceEnergyDensity (jkr.hpp:1369-1407), which runSimulation calls to turn the
// target equilibrium distance eqdist into the adhesion energy density (simulation.hpp:1354-1358).
// The reference nests two finite-difference Newton solves: the overlap where the JKR force
// 4 E0 a^3 / (3 Req) - 4 sqrt(pi gamma E0) a^(3/2) vanishes (jkr.hpp:1311-1339), inside a solve
// on log10(gamma).  The balance has a closed form.  Zero force means a^3 = 9 pi gamma Req^2 / E0,
// and the JKR overlap a^2 / Req - 2 sqrt(pi gamma a / E0) at that radius is
// (3 Req)^(1/3) (pi gamma / E0)^(2/3), so gamma = E0 delta^(3/2) / (pi sqrt(3 Req)) with
// delta = 2 R - eqdist.  The reference caps the overlap at 2 (R - Rcell), so a target below
// 2 Rcell, or at or above 2 R, has no solution.
int abm_jkr_optimal_gamma(double R, double Rcell, double E0, double eqdist, double* gamma)
{
    if (!gamma || !(R > 0) || !(E0 > 0) || !(Rcell >= 0) || !(Rcell < R)) return ABM_ERR_ARG;
    const double delta = 2 * R - eqdist;
    const double cap = 2 * (R - Rcell);
    if (!(delta > 0) || delta > cap * (1 + 4 * DBL_EPSILON)) return ABM_ERR_ARG;
    const double pi = 3.141592653589793238462643383279502884;
    *gamma = E0 * delta * std::sqrt(delta) / (pi * std::sqrt(3 * (R / 2)));
    return ABM_OK;
}

const char* abm_last_error(const abm_ctx* c) { return c ? c->err.c_str() : "null context"; }

static void free_all(abm_ctx* c)
{
    if (c->g_iter) cudaGraphExecDestroy(c->g_iter);
    if (c->g_iter_k) cudaGraphExecDestroy(c->g_iter_k);
    if (c->g_rebuild) cudaGraphExecDestroy(c->g_rebuild);
    void* ptrs[] = {c->geom, c->vel, c->phys, c->fcc, c->geom_c, c->vel_c, c->gen_tmp, c->k0buf, c->ctrl, c->grid,
                    c->bbox_acc, c->bbox_counter, c->bin_count, c->bin_start, c->key, c->slot,
                    c->sorted_cell, c->sorted_geom, c->scratch, c->nbr_count, c->row_ptr, c->col, c->lower_end, c->rev, c->pairs, c->pair_start, c->surv, c->jbuf,
                    c->scan_sums, c->jkr_delta, c->jkr_radius, c->jkr_gam, c->jkr_rad2, c->staging, c->div_flags, c->div_rank,
                    c->mothers, c->div_check, c->div_sat, c->div_ok, c->parents_dev, c->d1, c->d2, c->dlen,
                    c->dgrowth, c->mlp_w, c->log_buf, c->adhere, c->stat_part, c->order, c->order_flag,
                    c->order_pos, c->snap_geom, c->snap_vel, c->snap_phys, c->frame_info, c->phys_c, c->keep,
                    c->keep_rank, c->feta, c->fbuf, c->fmask, c->fr_list, c->ystage, c->snap_feta, c->pbuf,
                    c->whalf};
    for (void* q : ptrs) if (q) cudaFree(q);
    if (c->st) cudaStreamDestroy(c->st);
}

// the captured iteration graphs hold buffer pointers and parameters: drop them when
// those change (they are rebuilt at the next abm_iterate)
static void drop_iteration_graphs(abm_ctx* c)
{
    if (c->g_iter) { cudaGraphExecDestroy(c->g_iter); c->g_iter = nullptr; }
    if (c->g_iter_k) { cudaGraphExecDestroy(c->g_iter_k); c->g_iter_k = nullptr; }
}

static void fill_tableau(StepParams& sp, int mode, bool& ok)
{
    ok = true;
    memset(sp.A, 0, sizeof(sp.A)); memset(sp.b, 0, sizeof(sp.b)); memset(sp.bs, 0, sizeof(sp.bs));
    double q = 0;
    // simulation.hpp:1207-1268
    if (mode == ABM_HEUN_EULER)
    {
        sp.s = 2; sp.A[1][0] = 1; sp.b[0] = 0.5; sp.b[1] = 0.5; sp.bs[0] = 1; sp.bs[1] = 0; q = 1;
    }
    else if (mode == ABM_BOGACKI_SHAMPINE)
    {
        sp.s = 4;
        sp.A[1][0] = 1. / 2.; sp.A[2][1] = 3. / 4.; sp.A[3][0] = 2. / 9.; sp.A[3][1] = 1. / 3.; sp.A[3][2] = 4. / 9.;
        double b[4] = {2. / 9., 1. / 3., 4. / 9., 0}, bs[4] = {7. / 24., 1. / 4., 1. / 3., 1. / 8.};
        for (int i = 0; i < 4; ++i) { sp.b[i] = b[i]; sp.bs[i] = bs[i]; }
        q = 2;
    }
    else if (mode == ABM_RUNGE_KUTTA_FEHLBERG)
    {
        sp.s = 6;
        double A[6][6] = {{0, 0, 0, 0, 0, 0}, {1. / 4., 0, 0, 0, 0, 0}, {3. / 32., 9. / 32., 0, 0, 0, 0},
                          {1932. / 2197., -7200. / 2197., 7296. / 2197., 0, 0, 0},
                          {439. / 216., -8.0, 3680. / 513., -845. / 4104., 0, 0},
                          {-8. / 27., 2.0, -3544. / 2565., 1859. / 4104., -11. / 40., 0}};
        double b[6] = {16. / 135., 0, 6656. / 12825., 28561. / 56430., -9. / 50., 2. / 55.};
        double bs[6] = {25. / 216., 0, 1408. / 2565., 2197. / 4104., -1. / 5., 0};
        for (int i = 0; i < 6; ++i) { for (int j = 0; j < 6; ++j) sp.A[i][j] = A[i][j]; sp.b[i] = b[i]; sp.bs[i] = bs[i]; }
        q = 4;
    }
    else if (mode == ABM_DORMAND_PRINCE)
    {
        sp.s = 7;
        double A[7][7] = {{0, 0, 0, 0, 0, 0, 0}, {1. / 5., 0, 0, 0, 0, 0, 0}, {3. / 40., 9. / 40., 0, 0, 0, 0, 0},
                          {44. / 45., -56. / 15., 32. / 9., 0, 0, 0, 0},
                          {19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729, 0, 0, 0},
                          {9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656., 0, 0},
                          {35. / 384., 0, 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0}};
        double b[7] = {35. / 384., 0, 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0};
        double bs[7] = {5179. / 57600., 0, 7571. / 16695., 393. / 640., -92097. / 339200., 187. / 2100., 1. / 40.};
        for (int i = 0; i < 7; ++i) { for (int j = 0; j < 7; ++j) sp.A[i][j] = A[i][j]; sp.b[i] = b[i]; sp.bs[i] = bs[i]; }
        q = 4;
    }
    else ok = false;
    sp.inv_q1 = 1.0 / (q + 1);
}

__global__ void k_set_n(Ctrl* c, int n) { c->n = n; c->halted = 0; c->screen_valid = 0; c->n_order = 0; }
__global__ void k_screen_stale(Ctrl* c) { c->screen_valid = 0; }
__global__ void k_set_halt(Ctrl* c, int n_max) { c->halt_n = n_max; c->halted = 0; }
__global__ void k_set_clock(Ctrl* c, double t, double dt, int iter)
{
    c->t = t; c->dt = dt; c->iter = iter; c->mode = MODE_TRIAL; c->tries = 0; c->attempt = 0;
    c->err_bits = 0; c->blocks_done = 0;
}
__global__ void k_count_rebuild(Ctrl* c) { c->rebuilds += 1; }

int abm_create(const abm_params* q, abm_ctx** out)
{
    if (!q || !out) return ABM_ERR_ARG;
    *out = nullptr;
    abm_ctx* c = new abm_ctx();
    c->p = *q;
    abm_params& p = c->p;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
    {
        c->err = std::string("no CUDA device: ") + cudaGetErrorString(e);
        *out = c;
        return ABM_ERR_CUDA;
    }
    if (p.cap_cells <= 0 || p.R <= 0 || p.neighbor_threshold <= 0 || p.max_stepsize <= 0 ||
        p.iter_update_stepsize <= 0 || p.iter_update_neighbors <= 0)
    {
        c->err = "invalid parameters";
        *out = c;
        return ABM_ERR_ARG;
    }
    bool ok = true;
    c->verlet = p.integration_mode == ABM_VELOCITY_VERLET;
    if (c->verlet) { c->sp.s = 0; c->sp.inv_q1 = 0.0; }
    else fill_tableau(c->sp, p.integration_mode, ok);
    if (!ok) { c->err = "unsupported integration_mode"; *out = c; return ABM_ERR_ARG; }
    if (p.pair_lanes == 0) p.pair_lanes = 8;
    if (p.pair_lanes != 4 && p.pair_lanes != 8 && p.pair_lanes != 16 && p.pair_lanes != 32)
    {
        c->err = "pair_lanes must be 4, 8, 16 or 32"; *out = c; return ABM_ERR_ARG;
    }
    c->cap = p.cap_cells;
    // a compact 3-D colony reaches ~60 neighbors within the threshold (a 2-D monolayer ~30);
    // the defaults leave room above that, and overflow is reported, never truncated silently
    c->cap_nbr = p.cap_neighbors_per_cell > 0 ? p.cap_neighbors_per_cell : (p.dims == 2 ? 64 : 192);
    *out = c;
    CK(cudaGetDevice(&c->dev));
    CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->dev));
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    // bins: at least one per 2 cells, at most 4M
    c->cap_bins = std::min(std::max(c->cap * 2, 1 << 16), 1 << 22);
    const size_t cap = c->cap;
    CK(cudaMalloc(&c->geom, cap * sizeof(Geom)));
    CK(cudaMalloc(&c->vel, cap * sizeof(Vel)));
    CK(cudaMalloc(&c->phys, cap * sizeof(Phys)));
    CK(cudaMalloc(&c->fcc, cap * sizeof(Gen6)));
    CK(cudaMalloc(&c->geom_c, cap * sizeof(Geom)));
    CK(cudaMalloc(&c->vel_c, cap * sizeof(Vel)));
    CK(cudaMalloc(&c->gen_tmp, cap * sizeof(Gen6)));
    CK(cudaMalloc(&c->k0buf, cap * sizeof(Gen6)));
    CK(cudaMalloc(&c->ctrl, sizeof(Ctrl)));
    CK(cudaMalloc(&c->grid, sizeof(Grid)));
    CK(cudaMalloc(&c->bbox_acc, 8 * sizeof(unsigned long long)));
    CK(cudaMalloc(&c->bbox_counter, sizeof(unsigned int)));
    CK(cudaMalloc(&c->bin_count, (size_t)c->cap_bins * sizeof(int)));
    CK(cudaMalloc(&c->bin_start, ((size_t)c->cap_bins + 1) * sizeof(int)));
    CK(cudaMalloc(&c->key, cap * sizeof(int)));
    CK(cudaMalloc(&c->slot, cap * sizeof(int)));
    CK(cudaMalloc(&c->sorted_cell, cap * sizeof(int)));
    CK(cudaMalloc(&c->sorted_geom, cap * sizeof(Geom)));
    CK(cudaMalloc(&c->scratch, cap * c->cap_nbr * sizeof(int)));
    CK(cudaMalloc(&c->nbr_count, cap * sizeof(int)));
    CK(cudaMalloc(&c->row_ptr, (cap + 1) * sizeof(int)));
    CK(cudaMalloc(&c->col, cap * c->cap_nbr * sizeof(int)));
    CK(cudaMalloc(&c->lower_end, cap * sizeof(int)));
    CK(cudaMalloc(&c->rev, cap * c->cap_nbr * sizeof(int)));
    CK(cudaMalloc(&c->pairs, cap * c->cap_nbr / 2 * sizeof(int4) + sizeof(int4)));
    CK(cudaMalloc(&c->surv, cap * c->cap_nbr / 2 * sizeof(int) + sizeof(int)));
    CK(cudaMalloc(&c->pair_start, (cap + 1) * sizeof(int)));
    CK(cudaMalloc(&c->jbuf, cap * c->cap_nbr * sizeof(double4)));
    CK(cudaMemset(c->lower_end, 0, cap * sizeof(int)));
    size_t ns = std::max(scan_block_sums_size((int)cap + 1), scan_block_sums_size(c->cap_bins + 1)) + 1;
    CK(cudaMalloc(&c->scan_sums, ns * sizeof(int)));
    CK(cudaMalloc(&c->staging, cap * STAGING_COLS * sizeof(double)));
    CK(cudaMalloc(&c->div_flags, cap * sizeof(int)));
    CK(cudaMalloc(&c->div_rank, (cap + 1) * sizeof(int)));
    CK(cudaMalloc(&c->mothers, cap * sizeof(int)));
    CK(cudaMalloc(&c->div_check, cap * sizeof(int)));
    CK(cudaMalloc(&c->div_sat, cap * sizeof(int)));
    CK(cudaMalloc(&c->div_ok, 2 * cap * sizeof(int)));
    CK(cudaMalloc(&c->d1, cap * sizeof(Geom)));
    CK(cudaMalloc(&c->d2, cap * sizeof(Geom)));
    CK(cudaMalloc(&c->dlen, 2 * cap * sizeof(double)));
    CK(cudaMalloc(&c->dgrowth, 2 * cap * sizeof(double)));
    c->cap_parents = 2 * (int)cap + 1024;
    CK(cudaMalloc(&c->parents_dev, (size_t)c->cap_parents * sizeof(int)));
    CK(cudaMemset(c->row_ptr, 0, (cap + 1) * sizeof(int)));
    Ctrl h;
    memset(&h, 0, sizeof(h));
    h.dt = p.max_stepsize;
    h.mode = MODE_TRIAL;
    CK(cudaMemcpy(c->ctrl, &h, sizeof(Ctrl), cudaMemcpyHostToDevice));
    unsigned long long acc0[8] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
    CK(cudaMemcpy(c->bbox_acc, acc0, sizeof(acc0), cudaMemcpyHostToDevice));
    CK(cudaMemset(c->bbox_counter, 0, sizeof(unsigned int)));
    // parameters of the kernels
    MechParams mp;
    mp.R = p.R; mp.Rcell = p.Rcell; mp.E0 = p.E0; mp.Ecell = p.Ecell; mp.sqrtR = std::sqrt(p.R);
    mp.nz_threshold = p.nz_threshold; mp.coulomb = p.cell_surface_coulomb_coeff; mp.no_surface = p.no_surface;
    StepParams& sp = c->sp;
    sp.mp = mp;
    sp.tol = p.max_error_allowed; sp.min_error = p.min_error;
    sp.min_stepsize = p.min_stepsize; sp.max_stepsize = p.max_stepsize;
    sp.max_tries = p.max_tries_update_stepsize; sp.iter_update_stepsize = p.iter_update_stepsize;
    double nm[6] = {p.max_rxy_noise, p.max_rxy_noise, p.max_rz_noise, p.max_nxy_noise, p.max_nxy_noise, p.max_nz_noise};
    for (int k = 0; k < 6; ++k) sp.noise_max[k] = nm[k];
    sp.noise_on = (p.max_rxy_noise > 0 || p.max_rz_noise > 0 || p.max_nxy_noise > 0 || p.max_nz_noise > 0);
    sp.seed = p.rng_seed;
    sp.mixed = p.precision == ABM_PRECISION_MIXED && p.dims != 2;
    ForceParams& fp = c->fp;
    fp.R = p.R; fp.Rcell = p.Rcell; fp.E0 = p.E0;
    // simulation.hpp:1270-1274
    fp.pf0 = (4. / 3.) * p.E0 * std::sqrt(p.R / 2);
    fp.pf1 = (4. / 3.) * p.Ecell * std::sqrt(p.Rcell / 2);
    fp.pf2 = (4. / 3.) * p.E0 * std::sqrt(p.R / 2) * std::pow(2 * (p.R - p.Rcell), 1.5);
    fp.max_overlap = 2 * (p.R - p.Rcell);
    fp.adhesion = p.adhesion_mode != 0;
    fp.jkr_n = 0; fp.jkr_step = 1.0;
    fp.jkr_ng = 0; fp.jkr_gstep = 1.0; fp.jkr_gam = nullptr; fp.jkr_rad2 = nullptr;
    fp.skin = p.pair_skin == 0 ? 0.3 : std::max(p.pair_skin, 0.0);
    c->bp.threshold = p.neighbor_threshold;
    c->bp.prefilter = p.neighbor_threshold + p.Ldiv + 2 * p.R;
    c->bp.cap_per_cell = c->cap_nbr;
    DivideParams& dp = c->dp;
    dp.R = p.R; dp.Rcell = p.Rcell; dp.Ldiv = p.Ldiv;
    dp.growth_mean = p.growth_mean; dp.growth_std = p.growth_std;
    dp.daughter_length_std = p.daughter_length_std;
    dp.angle_xy_bound = p.daughter_angle_xy_bound; dp.angle_z_bound = p.daughter_angle_z_bound;
    dp.seed = p.rng_seed; dp.cap_cells = c->cap;
    dp.group_growth = 0; dp.inherit = 0; dp.n_start_switch = 0; dp.feta = nullptr;
    memset(&c->sw, 0, sizeof(c->sw));
    c->sw.seed = p.rng_seed; c->sw.R = p.R; c->sw.max_coord = 1;
    if (p.adhesion_mode != 0 && p.adhesion_mode != 1)
        return fail(c, ABM_ERR_ARG, "adhesion_mode must be 0 (none) or 1 (isotropic JKR, fixed gamma)");
    // 2-D model
    c->dims = (p.dims == 0) ? 3 : p.dims;
    if (c->dims != 2 && c->dims != 3) return fail(c, ABM_ERR_ARG, "dims must be 2 or 3");
    if (c->dims == 2)
    {
        if (p.integration_mode != ABM_HEUN_EULER && p.integration_mode != ABM_BOGACKI_SHAMPINE)
            return fail(c, ABM_ERR_ARG, "the 2-D model integrates with ABM_BOGACKI_SHAMPINE or ABM_HEUN_EULER");
        if (p.daughter_angle_z_bound != 0) return fail(c, ABM_ERR_ARG, "2-D daughters have no out-of-plane angle");
        if (p.precision != ABM_PRECISION_FP64) return fail(c, ABM_ERR_ARG, "the 2-D model runs in FP64");
        // 2D/include/simulation.hpp:232-237
        fp.pf2d[0] = 2.5 * p.E0 * std::sqrt(p.R);
        fp.pf2d[1] = 2.5 * p.E0 * std::sqrt(p.R) * std::pow(2 * (p.R - p.Rcell), 2.5);
        fp.pf2d[2] = 2.5 * p.Ecell * std::sqrt(p.Rcell);
        fp.adh_strength = p.adhesion_strength;
        fp.adh_mindist = p.adhesion_mindist;
        sp.rho_c = std::pow(p.sigma0 * p.R * p.R / (4 * p.E0), 1. / 3.);
        sp.max_noise_2d = p.max_noise;
        sp.noise_on = p.max_noise > 0;
        dp.angle_z_bound = 0.0;
        CK(cudaMalloc(&c->adhere, cap * c->cap_nbr));
        CK(cudaMemset(c->adhere, 0, cap * c->cap_nbr));
        fp.adhere = c->adhere;
    }
    // velocity Verlet (simulation.hpp:1279-1290, 1786-1798)
    if (c->verlet)
    {
        if (c->dims != 3) return fail(c, ABM_ERR_ARG, "velocity Verlet belongs to the 3-D model");
        if (p.precision != ABM_PRECISION_FP64) return fail(c, ABM_ERR_ARG, "velocity Verlet runs in FP64");
        if (p.controller != ABM_CONTROLLER_REFERENCE)
            return fail(c, ABM_ERR_ARG, "velocity Verlet takes a fixed step (reference controller)");
        if (!(p.M0 > 0)) return fail(c, ABM_ERR_ARG, "Initial cell mass must be defined when using velocity Verlet");
        c->rho = p.M0 / (M_PI * ((4. / 3.) * std::pow(p.R, 3) + p.R * p.R * p.L0));
        CK(cudaMalloc(&c->pbuf, cap * c->cap_nbr * sizeof(double4)));
        CK(cudaMalloc(&c->whalf, cap * sizeof(double4)));
    }
    // cell-cell kinetic friction (mechanics.hpp:1031-1175, 1339-1346)
    if (p.friction_mode != 0 && p.friction_mode != 1) return fail(c, ABM_ERR_ARG, "friction_mode must be 0 or 1");
    fp.fric = 0;
    sp.fric = 0;
    if (p.friction_mode == 1)
    {
        if (c->dims != 3) return fail(c, ABM_ERR_ARG, "cell-cell friction belongs to the 3-D model");
        if (p.precision != ABM_PRECISION_FP64) return fail(c, ABM_ERR_ARG, "cell-cell friction runs in FP64");
        c->eta_col = p.adhesion_mode != 0 ? 22 : 21;        // simulation.hpp:1184-1186
        const size_t ent = cap * c->cap_nbr;
        CK(cudaMalloc(&c->feta, cap * sizeof(double)));
        CK(cudaMemset(c->feta, 0, cap * sizeof(double)));
        CK(cudaMalloc(&c->fbuf, ent * sizeof(double4)));
        CK(cudaMalloc(&c->fmask, ent * sizeof(int)));
        CK(cudaMemset(c->fmask, 0, ent * sizeof(int)));
        CK(cudaMalloc(&c->fr_list, (ent / 2 + 1) * sizeof(int)));
        CK(cudaMalloc(&c->ystage, (size_t)MAX_STAGES * cap * sizeof(double2)));
        fp.fric = 1;
        fp.surface = !p.no_surface;
        fp.coulomb_cc = p.cell_cell_coulomb_coeff;
        fp.vel = c->vel;
        fp.feta = c->feta;
        fp.fbuf = c->fbuf;
        fp.fmask = c->fmask;
        fp.fr_list = c->fr_list;
        sp.fric = 1;
        c->dp.feta = c->feta;
    }
    if (p.controller != ABM_CONTROLLER_REFERENCE && p.controller != ABM_CONTROLLER_LEARNED &&
        p.controller != ABM_CONTROLLER_PI)
        return fail(c, ABM_ERR_ARG, "controller must be ABM_CONTROLLER_REFERENCE, _LEARNED or _PI");
    if (p.stepsize_log_capacity < 0) return fail(c, ABM_ERR_ARG, "stepsize_log_capacity must be >= 0");
    // step-size network, its features and the feature log
    sp.network = p.controller == ABM_CONTROLLER_LEARNED;
    sp.pi = p.controller == ABM_CONTROLLER_PI;
    sp.propose = sp.network || sp.pi;
    sp.log_cap = p.stepsize_log_capacity;
    sp.stats_on = sp.network || sp.log_cap > 0;
    sp.near_div_length = 0.9 * p.Ldiv;
    fp.stats = sp.stats_on;
    CK(cudaMalloc(&c->mlp_w, MLP_NPARAM * sizeof(float)));
    CK(cudaMemset(c->mlp_w, 0, MLP_NPARAM * sizeof(float)));
    if (sp.log_cap > 0)
    {
        CK(cudaMalloc(&c->log_buf, (size_t)sp.log_cap * MLP_LOG_COLS * sizeof(float)));
        CK(cudaMemset(c->log_buf, 0, (size_t)sp.log_cap * MLP_LOG_COLS * sizeof(float)));
    }
    sp.log_buf = c->log_buf;
    CK(cudaMalloc(&c->stat_part, (size_t)attempt_blocks(c->cap) * sizeof(double4)));
    sp.stat_part = c->stat_part;
    if (c->dims == 3)
    {
        CK(cudaMalloc(&c->order, (size_t)c->cap * sizeof(int)));
        CK(cudaMalloc(&c->order_flag, ((size_t)c->cap + 1) * sizeof(int)));
        CK(cudaMalloc(&c->order_pos, ((size_t)c->cap + 1) * sizeof(int)));
    }
    sp.order = c->order;
    return ABM_OK;
}

int abm_destroy(abm_ctx* c)
{
    if (!c) return ABM_ERR_ARG;
    if (c->st) cudaStreamSynchronize(c->st);
    free_all(c);
    delete c;
    return ABM_OK;
}

int abm_get_stream(abm_ctx* c, void** stream)
{
    if (!c || !stream) return ABM_ERR_ARG;
    *stream = (void*)c->st;
    return ABM_OK;
}

static int check_status(abm_ctx* c)
{
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (h.status & ST_NAN) return fail(c, ABM_ERR_NAN, "NaN/Inf in the RK error norm or velocities");
    if (h.status & ST_NBR_OVERFLOW) return fail(c, ABM_ERR_CAPACITY, "neighbors per cell exceed cap_neighbors_per_cell");
    if (h.status & ST_BIN_OVERFLOW) return fail(c, ABM_ERR_CAPACITY, "cell-list grid exceeds the bin capacity");
    if (h.status & ST_CELL_OVERFLOW) return fail(c, ABM_ERR_CAPACITY, "division exceeds cap_cells");
    return ABM_OK;
}

int abm_synchronize(abm_ctx* c)
{
    if (!c) return ABM_ERR_ARG;
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());
    return check_status(c);
}

static void drop_variable_table(abm_ctx* c)
{
    if (c->jkr_gam) { cudaFree(c->jkr_gam); cudaFree(c->jkr_rad2); c->jkr_gam = c->jkr_rad2 = nullptr; }
    c->fp.jkr_ng = 0; c->fp.jkr_gam = nullptr; c->fp.jkr_rad2 = nullptr;
}

int abm_set_jkr_table(abm_ctx* c, const double* delta, const double* radius, int n)
{
    if (!c || !delta || !radius || n < 2 || n > 512) return fail(c, ABM_ERR_ARG, "JKR table needs 2..512 entries");
    for (int i = 1; i < n; ++i)
        if (!(delta[i] > delta[i - 1])) return fail(c, ABM_ERR_ARG, "JKR overlap mesh must be increasing");
    drop_variable_table(c);
    if (c->jkr_delta) { cudaFree(c->jkr_delta); cudaFree(c->jkr_radius); c->jkr_delta = c->jkr_radius = nullptr; }
    CK(cudaMalloc(&c->jkr_delta, n * sizeof(double)));
    CK(cudaMalloc(&c->jkr_radius, n * sizeof(double)));
    CK(cudaMemcpy(c->jkr_delta, delta, n * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->jkr_radius, radius, n * sizeof(double), cudaMemcpyHostToDevice));
    c->jkr_n = n;
    c->fp.jkr_n = n;
    c->fp.jkr_step = (delta[n - 1] - delta[0]) / double(n - 1);
    drop_iteration_graphs(c);
    return ABM_OK;
}

int abm_set_jkr_table_variable(abm_ctx* c, const double* delta, int n_delta, const double* gamma, int n_gamma,
                               const double* radius)
{
    if (!c) return ABM_ERR_ARG;
    if (!delta || !gamma || !radius || n_gamma < 2 || n_gamma > 4096)
        return fail(c, ABM_ERR_ARG, "variable JKR table needs 2..512 overlaps and 2..4096 gammas");
    for (int j = 1; j < n_gamma; ++j)
        if (!(gamma[j] > gamma[j - 1])) return fail(c, ABM_ERR_ARG, "JKR gamma mesh must be increasing");
    if (!(gamma[0] >= 0)) return fail(c, ABM_ERR_ARG, "JKR gamma mesh must start at gamma >= 0");
    // the fixed-gamma slots hold the overlap mesh and the radii at the largest gamma
    std::vector<double> last((size_t)std::max(n_delta, 0));
    for (int i = 0; i < n_delta; ++i) last[i] = radius[(size_t)i * n_gamma + (n_gamma - 1)];
    int rc = abm_set_jkr_table(c, delta, last.data(), n_delta);
    if (rc) return rc;
    CK(cudaMalloc(&c->jkr_gam, (size_t)n_gamma * sizeof(double)));
    CK(cudaMalloc(&c->jkr_rad2, (size_t)n_delta * n_gamma * sizeof(double)));
    CK(cudaMemcpy(c->jkr_gam, gamma, (size_t)n_gamma * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->jkr_rad2, radius, (size_t)n_delta * n_gamma * sizeof(double), cudaMemcpyHostToDevice));
    c->fp.jkr_ng = n_gamma;
    c->fp.jkr_gstep = (gamma[n_gamma - 1] - gamma[0]) / double(n_gamma - 1);
    c->fp.jkr_gam = c->jkr_gam;
    c->fp.jkr_rad2 = c->jkr_rad2;
    drop_iteration_graphs(c);
    return ABM_OK;
}

// switching moves cells between growth-rate distributions: division is possible when
// either group's distribution is not the zero rate
static bool switch_grows(const abm_ctx* c)
{
    const SwitchParams& w = c->sw;
    return w.mode != 0 && (w.gmean[0] != 0 || w.gmean[1] != 0 || w.gstd[0] != 0 || w.gstd[1] != 0);
}

static int ensure_post_buffers(abm_ctx* c)
{
    if (!c->keep) CK(cudaMalloc(&c->keep, (size_t)c->cap * sizeof(int)));
    if (!c->keep_rank) CK(cudaMalloc(&c->keep_rank, ((size_t)c->cap + 1) * sizeof(int)));
    if (!c->phys_c) CK(cudaMalloc(&c->phys_c, (size_t)c->cap * sizeof(Phys)));
    return ABM_OK;
}

static void update_post(abm_ctx* c)
{
    const bool on = c->sw.mode != 0 || c->sw.basal;
    if (on != c->post_on) drop_iteration_graphs(c);
    c->post_on = on;
    if (switch_grows(c) && !c->div_enabled) { c->div_enabled = true; drop_iteration_graphs(c); }
}

int abm_set_switching(abm_ctx* c, int mode, int n_start, const double* rates, const double* growth_mean,
                      const double* growth_std, double timescale, int n_attr, const int* attr_col,
                      const double* attr_targets, double max_gamma, int modulate, const double* visc_lims,
                      int max_coord)
{
    if (!c) return ABM_ERR_ARG;
    if (c->dims != 3) return fail(c, ABM_ERR_STATE, "switching belongs to the 3-D model");
    if (mode < 0 || mode > 2) return fail(c, ABM_ERR_ARG, "switching mode must be 0 (none), 1 (Markov) or 2 (inherit)");
    if (mode != 0 && (!rates || !growth_mean || !growth_std))
        return fail(c, ABM_ERR_ARG, "switching needs rates and growth distributions");
    if (n_attr < 0 || n_attr > 4 || (n_attr > 0 && (!attr_col || !attr_targets)))
        return fail(c, ABM_ERR_ARG, "0..4 switched attributes, with columns and targets");
    if (!(timescale >= 0) || !(max_gamma >= 0) || max_coord < 1)
        return fail(c, ABM_ERR_ARG, "timescale and max_gamma must be >= 0, max_coord >= 1");
    if (modulate && !visc_lims) return fail(c, ABM_ERR_ARG, "local viscosity needs its limits");
    SwitchParams& w = c->sw;
    w.mode = mode;
    w.n_start = n_start;
    for (int k = 0; k < 4; ++k) w.rates[k] = mode != 0 ? rates[k] : 0.0;
    for (int g = 0; g < 2; ++g)
    {
        w.gmean[g] = mode != 0 ? growth_mean[g] : 0.0;
        w.gstd[g] = mode != 0 ? growth_std[g] : 0.0;
    }
    for (int k = 0; k < 4; ++k)
        if (!(w.rates[k] >= 0) || !std::isfinite(w.rates[k])) return fail(c, ABM_ERR_ARG, "rates must be finite and >= 0");
    w.timescale = timescale;
    w.n_attr = n_attr;
    for (int k = 0; k < n_attr; ++k)
    {
        // the reference's drivers switch eta0, eta1 and sigma0 (indices.hpp: columns 17-19)
        if (attr_col[k] < 17 || attr_col[k] > 19)
            return fail(c, ABM_ERR_ARG, "switched attributes are columns 17 (eta0), 18 (eta1) or 19 (sigma0)");
        w.attr_field[k] = attr_col[k] - 15;          // Phys: l, growth, eta0, eta1, sigma0, ...
        w.target[0][k] = attr_targets[k];
        w.target[1][k] = attr_targets[n_attr + k];
    }
    w.max_gamma = max_gamma;
    w.gamma_ramp = mode != 0 && c->p.adhesion_mode != 0;
    w.modulate = (mode != 0 && c->p.adhesion_mode != 0 && modulate) ? 1 : 0;
    for (int k = 0; k < 4; ++k) w.visc[k] = visc_lims ? visc_lims[k] : 0.0;
    w.max_coord = max_coord;
    // division: the daughters' growth rates follow the mother's group, and inherited
    // switching acts on each pair of daughters
    DivideParams& dp = c->dp;
    dp.group_growth = mode != 0;
    for (int g = 0; g < 2; ++g) { dp.gmean[g] = w.gmean[g]; dp.gstd[g] = w.gstd[g]; }
    dp.inherit = mode == 2;
    dp.n_start_switch = n_start;
    for (int k = 0; k < 4; ++k) dp.rates[k] = w.rates[k];
    if (mode != 0)
    {
        int rc = ensure_post_buffers(c);
        if (rc) return rc;
    }
    drop_iteration_graphs(c);                 // the parameters are baked into the graph's nodes
    update_post(c);
    return ABM_OK;
}

int abm_set_basal_only(abm_ctx* c, int basal_only, double min_overlap)
{
    if (!c) return ABM_ERR_ARG;
    if (c->dims != 3) return fail(c, ABM_ERR_STATE, "basal-only compaction belongs to the 3-D model");
    if (!std::isfinite(min_overlap)) return fail(c, ABM_ERR_ARG, "min_overlap must be finite");
    // simulation.hpp:1831: only with the surface present
    c->sw.basal = (basal_only && !c->p.no_surface) ? 1 : 0;
    c->sw.basal_min_overlap = min_overlap;
    if (c->sw.basal)
    {
        int rc = ensure_post_buffers(c);
        if (rc) return rc;
    }
    drop_iteration_graphs(c);
    update_post(c);
    return ABM_OK;
}

int abm_basal_dropped(abm_ctx* c, long long* dropped)
{
    if (!c || !dropped) return ABM_ERR_ARG;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *dropped = h.basal_dropped;
    return ABM_OK;
}

int abm_upload_cells(abm_ctx* c, const double* cm, int n, int ncols, int ld)
{
    if (!c || !cm || n < 0 || ld < n) return fail(c, ABM_ERR_ARG, "bad cell array");
    if (n > c->cap) return fail(c, ABM_ERR_CAPACITY, "more cells than cap_cells");
    const bool two_d = c->dims == 2;
    if (two_d && (ncols < 17 || ncols > STAGING_COLS)) return fail(c, ABM_ERR_ARG, "2-D cell arrays need 17..32 columns");
    if (!two_d && (ncols < 21 || ncols > STAGING_COLS)) return fail(c, ABM_ERR_ARG, "cell arrays need 21..32 columns");
    if (!two_d && c->p.adhesion_mode != 0 && ncols < 22)
        return fail(c, ABM_ERR_ARG, "adhesion needs the gamma column (21)");
    if (c->sp.fric && ncols <= c->eta_col)
        return fail(c, ABM_ERR_ARG, "friction needs the cell-cell friction column (22 with adhesion, 21 without)");
    c->ncols = ncols;
    // the gamma column travels with the cells when present (used with adhesion only)
    c->has_gamma = !two_d && ncols > 21;
    if (n > 0)
    {
        CK(cudaMemcpy2DAsync(c->staging, (size_t)n * sizeof(double), cm, (size_t)ld * sizeof(double),
                             (size_t)n * sizeof(double), ncols, cudaMemcpyHostToDevice, c->st));
        if (two_d) launch_cells_from_colmajor_2d(c->staging, n, ncols, n, c->geom, c->vel, c->phys, c->st);
        else launch_cells_from_colmajor(c->staging, n, ncols, n, c->has_gamma, c->geom, c->vel, c->phys, c->st);
        if (c->sp.fric)
            CK(cudaMemcpyAsync(c->feta, c->staging + (size_t)c->eta_col * n, (size_t)n * sizeof(double),
                               cudaMemcpyDeviceToDevice, c->st));
    }
    k_set_n<<<1, 1, 0, c->st>>>(c->ctrl, n);
    CK(cudaGetLastError());
    if (c->n_host != n) c->nbrs_valid = false;
    c->n_host = n;
    c->cells_loaded = true;
    // division is possible when a cell already exceeds Ldiv or any cell can grow
    bool grows = (c->p.growth_mean != 0 || c->p.growth_std != 0) || switch_grows(c);
    const int col_growth = two_d ? 12 : 16, col_l = two_d ? 9 : 13;
    for (int i = 0; i < n && !grows; ++i)
        grows = cm[(size_t)col_growth * ld + i] != 0 || cm[(size_t)col_l * ld + i] > c->p.Ldiv;
    if (grows != c->div_enabled) drop_iteration_graphs(c);
    c->div_enabled = grows;
    return ABM_OK;
}

// friction: the coefficient column of a column-major staging copy of n cells
static int stage_eta_column(abm_ctx* c, const double* src, int n)
{
    if (c->sp.fric && c->ncols > c->eta_col && n > 0)
        CK(cudaMemcpyAsync(c->staging + (size_t)c->eta_col * n, src, (size_t)n * sizeof(double),
                           cudaMemcpyDeviceToDevice, c->st));
    return ABM_OK;
}

int abm_download_cells(abm_ctx* c, double* cm, int ld)
{
    if (!c || !cm) return ABM_ERR_ARG;
    if (!c->cells_loaded) return fail(c, ABM_ERR_STATE, "no cells uploaded");
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int n = h.n;
    c->n_host = n;
    if (ld < n) return fail(c, ABM_ERR_ARG, "ld smaller than the cell count");
    if (n > 0)
    {
        if (c->dims == 2) launch_cells_to_colmajor_2d(c->geom, c->vel, c->phys, n, c->ncols, n, c->staging, c->st);
        else launch_cells_to_colmajor(c->geom, c->vel, c->phys, n, c->ncols, n, c->has_gamma, c->staging, c->st);
        int rc = stage_eta_column(c, c->feta, n);
        if (rc) return rc;
        CK(cudaMemcpy2DAsync(cm, (size_t)ld * sizeof(double), c->staging, (size_t)n * sizeof(double),
                             (size_t)n * sizeof(double), c->ncols, cudaMemcpyDeviceToHost, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return ABM_OK;
}

// frames (simulation.hpp:2025-2058): dt_write > 0 and slots > 0 turn them on
__global__ void k_set_frames(Ctrl* c, double dt_write)
{
    c->dt_write = dt_write;
    c->frame_due = 0;
    c->frames_taken = 0;
    c->frame_blocks = 0u;
}

int abm_set_frames(abm_ctx* c, double dt_write, int slots)
{
    if (!c || slots < 0 || !(dt_write >= 0)) return ABM_ERR_ARG;
    const bool on = dt_write > 0 && slots > 0;
    if (!on) slots = 0;
    if (slots != c->frame_slots)
    {
        CK(cudaStreamSynchronize(c->st));
        cudaFree(c->snap_geom); cudaFree(c->snap_vel); cudaFree(c->snap_phys); cudaFree(c->frame_info);
        cudaFree(c->snap_feta);
        c->snap_geom = nullptr; c->snap_vel = nullptr; c->snap_phys = nullptr; c->frame_info = nullptr;
        c->snap_feta = nullptr;
        if (slots > 0)
        {
            const size_t m = (size_t)slots * c->cap;
            CK(cudaMalloc(&c->snap_geom, m * sizeof(Geom)));
            CK(cudaMalloc(&c->snap_vel, m * sizeof(Vel)));
            CK(cudaMalloc(&c->snap_phys, m * sizeof(Phys)));
            CK(cudaMalloc(&c->frame_info, (size_t)slots * sizeof(FrameInfo)));
            if (c->sp.fric) CK(cudaMalloc(&c->snap_feta, m * sizeof(double)));
        }
        c->frame_slots = slots;
        drop_iteration_graphs(c);          // the snapshot is a node of the iteration graph
    }
    k_set_frames<<<1, 1, 0, c->st>>>(c->ctrl, on ? dt_write : 0.0);
    CK(cudaGetLastError());
    return ABM_OK;
}

int abm_frames_taken(abm_ctx* c, int* taken)
{
    if (!c || !taken) return ABM_ERR_ARG;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *taken = h.frames_taken;
    return ABM_OK;
}

int abm_download_frame(abm_ctx* c, int index, double* cm, int ld, int* n, double* t, int* iter, int* n_parents)
{
    if (!c || !n || index < 0) return ABM_ERR_ARG;
    if (c->frame_slots <= 0) return fail(c, ABM_ERR_STATE, "frames are off (abm_set_frames)");
    int taken = 0;
    int rc = abm_frames_taken(c, &taken);
    if (rc) return rc;
    if (index >= taken) return fail(c, ABM_ERR_ARG, "no such frame yet");
    if (index < taken - c->frame_slots)
        return fail(c, ABM_ERR_CAPACITY, "the frame was overwritten: download frames more often or use more slots");
    const int slot = index % c->frame_slots;
    FrameInfo f;
    CK(cudaMemcpy(&f, c->frame_info + slot, sizeof(FrameInfo), cudaMemcpyDeviceToHost));
    *n = f.n;
    if (t) *t = f.t;
    if (iter) *iter = f.iter;
    if (n_parents) *n_parents = f.n_parents;
    if (!cm) return ABM_OK;                 // sizes only
    if (ld < f.n) return fail(c, ABM_ERR_ARG, "ld smaller than the frame's cell count");
    if (f.n > 0)
    {
        const size_t off = (size_t)slot * c->cap;
        if (c->dims == 2)
            launch_cells_to_colmajor_2d(c->snap_geom + off, c->snap_vel + off, c->snap_phys + off, f.n, c->ncols,
                                        f.n, c->staging, c->st);
        else
            launch_cells_to_colmajor(c->snap_geom + off, c->snap_vel + off, c->snap_phys + off, f.n, c->ncols, f.n,
                                     c->has_gamma, c->staging, c->st);
        if (c->snap_feta)
        {
            rc = stage_eta_column(c, c->snap_feta + off, f.n);
            if (rc) return rc;
        }
        CK(cudaMemcpy2DAsync(cm, (size_t)ld * sizeof(double), c->staging, (size_t)f.n * sizeof(double),
                             (size_t)f.n * sizeof(double), c->ncols, cudaMemcpyDeviceToHost, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return ABM_OK;
}

int abm_get_num_cells(abm_ctx* c, int* n)
{
    if (!c || !n) return ABM_ERR_ARG;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *n = h.n;
    return ABM_OK;
}

int abm_set_clock(abm_ctx* c, double t, double dt, int iter)
{
    if (!c || !(dt > 0)) return ABM_ERR_ARG;
    k_set_clock<<<1, 1, 0, c->st>>>(c->ctrl, t, dt, iter);
    CK(cudaGetLastError());
    c->host_iter = iter;
    return ABM_OK;
}

int abm_get_clock(abm_ctx* c, double* t, double* dt, int* iter)
{
    if (!c) return ABM_ERR_ARG;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (t) *t = h.t;
    if (dt) *dt = h.dt;
    if (iter) *iter = h.iter;
    return ABM_OK;
}

__global__ void k_set_n_parents(Ctrl* c, int n) { c->n_parents = n; }

int abm_set_parents(abm_ctx* c, const int* parents, int n)
{
    if (!c || (n > 0 && !parents) || n < 0) return ABM_ERR_ARG;
    // room for the given lineage plus two entries per division up to cap_cells cells
    if ((long long)n + 2LL * c->cap > (long long)c->cap_parents)
    {
        CK(cudaStreamSynchronize(c->st));
        CK(cudaFree(c->parents_dev));
        c->parents_dev = nullptr;
        c->cap_parents = n + 2 * c->cap + 1024;
        CK(cudaMalloc(&c->parents_dev, (size_t)c->cap_parents * sizeof(int)));
        // captured graphs hold the old buffer
        drop_iteration_graphs(c);
        if (c->g_rebuild) { cudaGraphExecDestroy(c->g_rebuild); c->g_rebuild = nullptr; }
    }
    if (n > 0) CK(cudaMemcpyAsync(c->parents_dev, parents, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, c->st));
    k_set_n_parents<<<1, 1, 0, c->st>>>(c->ctrl, n);
    CK(cudaStreamSynchronize(c->st));
    return ABM_OK;
}

int abm_get_parents(abm_ctx* c, int* out, int cap, int* n)
{
    if (!c) return ABM_ERR_ARG;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (n) *n = h.n_parents;
    if (out && h.n_parents > 0)
        CK(cudaMemcpy(out, c->parents_dev, (size_t)std::min(cap, h.n_parents) * sizeof(int), cudaMemcpyDeviceToHost));
    return ABM_OK;
}

// neighbor rebuild sequence (getCellNeighbors, mechanics.hpp:520-593)
static void enqueue_rebuild(abm_ctx* c)
{
    cudaStream_t st = c->st;
    launch_bbox(c->geom, c->ctrl, c->grid, c->bbox_acc, c->bbox_counter, c->bp.prefilter, c->cap_bins, c->cap, st);
    cudaMemsetAsync(c->bin_count, 0, (size_t)c->cap_bins * sizeof(int), st);
    launch_bin_count(c->geom, c->ctrl, c->grid, c->bin_count, c->key, c->slot, c->cap, st);
    launch_scan(c->bin_count, &c->grid->nbins, c->bin_start, c->scan_sums, c->cap_bins, st);
    launch_bin_scatter(c->geom, c->ctrl, c->bin_start, c->key, c->slot, c->sorted_cell, c->sorted_geom, c->cap, st);
    launch_pair_build(c->grid, c->bin_start, c->sorted_cell, c->sorted_geom, c->ctrl, c->bp, c->scratch,
                      c->nbr_count, c->cap_bins, c->num_sms, st);
    launch_scan(c->nbr_count, &c->ctrl->n, c->row_ptr, c->scan_sums, c->cap, st);
    launch_csr_fill(c->ctrl, c->row_ptr, c->scratch, c->cap_nbr, c->col, c->ctrl, c->cap, st);
    launch_csr_rev(c->ctrl, c->row_ptr, c->col, c->lower_end, c->rev, c->cap, st);
    // pairs in the bin order of the sort just made (sorted_cell)
    launch_pair_list(c->ctrl, c->row_ptr, c->lower_end, c->col, c->rev, c->nbr_count, c->pair_start, c->scan_sums,
                     c->pairs, c->cap, st, c->sorted_cell);
    if (c->dims == 2 && c->p.adhesion_mode != 0)
        launch_adhere_flags(c->ctrl, c->row_ptr, c->col, c->geom, c->p.R, c->p.Rcell, c->adhere, c->cap, st);
    if (c->order)
        launch_attempt_order(c->geom, c->ctrl, c->sp.mp, c->order_flag, c->order_pos, c->scan_sums, c->order,
                             c->cap, st);
    k_count_rebuild<<<1, 1, 0, st>>>(c->ctrl);
}

// one iteration of the loop body without division: stage-invariant pair
// forces, then the trial attempt, up to max_tries retries and the accepted
// final attempt (simulation.hpp:1677-1769), each an early exit when idle
// the screened pass writes both shares of every pair; with_gather also sums them
// per cell into fcc (the API paths; the loop's first attempt sums them itself)
// in_loop: the pass of a loop iteration, one of whose blocks also makes the iteration's
// step-size features (and, learned, the proposed dt)
static void enqueue_pair_force(abm_ctx* c, int with_gather, bool in_loop = false)
{
    launch_pair_screened(c->geom, c->row_ptr, c->lower_end, c->col, c->rev, c->ctrl, c->fp,
                         c->jkr_delta, c->jkr_radius, c->fcc, c->jbuf, c->p.precision == ABM_PRECISION_MIXED,
                         c->cap * c->cap_nbr, c->cap, c->num_sms, c->st, with_gather, c->dims, c->p.pair_tile,
                         c->p.pair_blocks_per_sm, c->pairs, c->surv, in_loop ? &c->sp : nullptr, c->mlp_w);
}

// pair_sum 1 (default): the first attempt sums each cell's shares itself; 2: a
// separate light kernel sums them into fcc before the attempts
static bool sum_in_attempt(abm_ctx* c) { return c->p.pair_sum != 2; }

// the loop's pair pass: the shares, plus their per-cell sums unless the first attempt
// makes them, and the step-size proposal
static void enqueue_loop_pair_force(abm_ctx* c) { enqueue_pair_force(c, sum_in_attempt(c) ? 0 : 1, true); }

// where the attempts of one iteration find the pair force
static PairGather loop_gather(abm_ctx* c)
{
    const bool f32 = c->p.precision == ABM_PRECISION_MIXED && c->dims == 3;
    PairGather pg = {sum_in_attempt(c) ? (f32 ? 3 : 2) : 0, c->row_ptr, c->lower_end, c->jbuf, c->fcc,
                     c->fbuf, c->fmask, c->ystage, c->cap};
    return pg;
}

// friction with a surface: the trial passes and decision checks that precede an attempt
// of kind `kind` (no candidates without a surface)
static void enqueue_friction_rounds(abm_ctx* c, int kind, PairGather pg, double eval_dt = 0.0, int eval_attempt = 0)
{
    if (!c->sp.fric || !c->fp.surface || c->verlet) return;
    launch_friction_rounds(kind, c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->geom_c, c->vel_c, c->k0buf,
                           eval_dt, eval_attempt, c->cap, c->st, pg, c->pairs, c->fr_list, c->fmask, c->p.R);
}


// one velocity-Verlet step (integration mode 0) at the context's dt, growth included
static void enqueue_verlet_step(abm_ctx* c)
{
    launch_verlet_step(c->geom, c->vel, c->phys, c->geom_c, c->vel_c, c->whalf, c->ctrl, c->sp, c->fp,
                       c->jkr_delta, c->jkr_radius, c->pairs, c->row_ptr, c->lower_end, c->jbuf, c->pbuf, c->rho,
                       c->cap, c->cap * c->cap_nbr / 2, c->st);
}

static void enqueue_attempts(abm_ctx* c)
{
    cudaStream_t st = c->st;
    PairGather pg = loop_gather(c);
    enqueue_friction_rounds(c, MODE_TRIAL, pg);
    launch_attempt(MODE_TRIAL, c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->geom_c, c->vel_c, nullptr,
                   c->k0buf, 0.0, 0, c->cap, st, 0, 0, pg, c->dims);
    for (int r = 0; r < c->p.max_tries_update_stepsize; ++r)
    {
        enqueue_friction_rounds(c, MODE_RETRY, pg);
        launch_attempt(MODE_RETRY, c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->geom_c, c->vel_c, nullptr,
                       c->k0buf, 0.0, 0, c->cap, st, 0, 0, pg, c->dims);
    }
    enqueue_friction_rounds(c, MODE_FINAL, pg);
    launch_attempt(MODE_FINAL, c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->geom_c, c->vel_c, nullptr,
                   c->k0buf, 0.0, 0, c->cap, st, 0, 0, pg, c->dims);
}

// the snapshot of a frame marked by this iteration's accepted step (frames enabled)
static void enqueue_frame_snapshot(abm_ctx* c)
{
    launch_frame_snapshot(c->geom, c->vel, c->phys, c->ctrl, c->snap_geom, c->snap_vel, c->snap_phys,
                          c->frame_info, c->frame_slots, c->cap, c->st, c->sp.fric ? c->feta : nullptr,
                          c->snap_feta);
}

static void enqueue_iteration(abm_ctx* c)
{
    if (c->verlet) enqueue_verlet_step(c);
    else
    {
        enqueue_loop_pair_force(c);
        enqueue_attempts(c);
    }
    if (c->frame_slots > 0) enqueue_frame_snapshot(c);
}

static int capture(abm_ctx* c, void (*fn)(abm_ctx*), cudaGraphExec_t* exec)
{
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    fn(c);
    CK(cudaStreamEndCapture(c->st, &g));
    cudaError_t inst_plain = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    CK(inst_plain);
    return ABM_OK;
}

// division body (after the flag count): ranks, room checks on a fresh cell list,
// the ten tries, commit, then the neighbor rebuild the reference does after any
// division (simulation.hpp:1654-1660)
// the body up to the room checks (before the tries)
static void enqueue_division_setup(abm_ctx* c)
{
    cudaStream_t st = c->st;
    launch_scan(c->div_flags, &c->ctrl->n, c->div_rank, c->scan_sums, c->cap, st);
    launch_div_body_pre(c->ctrl, c->div_flags, c->div_rank, c->mothers, c->cap, st);
    launch_bbox(c->geom, c->ctrl, c->grid, c->bbox_acc, c->bbox_counter, c->bp.prefilter, c->cap_bins, c->cap, st);
    cudaMemsetAsync(c->bin_count, 0, (size_t)c->cap_bins * sizeof(int), st);
    launch_bin_count(c->geom, c->ctrl, c->grid, c->bin_count, c->key, c->slot, c->cap, st);
    launch_scan(c->bin_count, &c->grid->nbins, c->bin_start, c->scan_sums, c->cap_bins, st);
    launch_bin_scatter(c->geom, c->ctrl, c->bin_start, c->key, c->slot, c->sorted_cell, c->sorted_geom, c->cap, st);
    launch_div_check(c->geom, c->ctrl, c->dp, c->grid, c->bin_start, c->sorted_cell, c->sorted_geom, c->div_flags,
                     c->mothers, c->div_check, c->div_sat, st);
}

static void enqueue_division_commit(abm_ctx* c)
{
    launch_div_commit(c->geom, c->vel, c->phys, c->ctrl, c->dp, c->mothers, c->d1, c->d2, c->dlen, c->dgrowth,
                      c->parents_dev, c->st);
}

// the whole body with the ten tries launched in a row (each exits at once once the
// criterion holds for every dividing cell): the paths without conditional nodes
static void enqueue_division_body(abm_ctx* c)
{
    enqueue_division_setup(c);
    launch_div_tries(c->geom, c->phys, c->ctrl, c->dp, c->grid, c->bin_start, c->sorted_cell, c->sorted_geom,
                     c->div_flags, c->mothers, c->div_check, c->div_sat, c->d1, c->d2, c->dlen, c->dgrowth,
                     c->div_ok, c->st);
    enqueue_division_commit(c);
}

// Capture fn into `graph` after `deps`; `deps` becomes the leaf set of the capture.
static int capture_into(abm_ctx* c, cudaGraph_t graph, std::vector<cudaGraphNode_t>& deps,
                        const std::function<void()>& fn)
{
    CK(cudaStreamBeginCaptureToGraph(c->st, graph, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                     cudaStreamCaptureModeThreadLocal));
    fn();
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t* leaves = nullptr;
    size_t nleaves = 0;
    cudaError_t info = cudaStreamGetCaptureInfo(c->st, &status, nullptr, nullptr, &leaves, &nleaves);
    std::vector<cudaGraphNode_t> next(leaves, leaves + (info == cudaSuccess ? nleaves : 0));
    CK(cudaStreamEndCapture(c->st, nullptr));
    CK(info);
    deps = next;
    return ABM_OK;
}

static int add_conditional(abm_ctx* c, cudaGraph_t graph, std::vector<cudaGraphNode_t>& deps,
                           cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                           cudaGraph_t* body)
{
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams* np = reinterpret_cast<cudaGraphNodeParams*>(raw);
    np->type = cudaGraphNodeTypeConditional;
    np->conditional.handle = h;
    np->conditional.type = type;
    np->conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, graph, deps.empty() ? nullptr : deps.data(), deps.size(), np));
    *body = np->conditional.phGraph_out[0];
    deps.assign(1, node);
    return ABM_OK;
}

// the body in a graph: the tries as a WHILE node that runs them until the distance
// criterion holds for every dividing cell or ten have run (growth.hpp:252), then the
// commit and the neighbor rebuild
static int capture_division_body(abm_ctx* c, cudaGraph_t body)
{
    std::vector<cudaGraphNode_t> bd;
    int rc = capture_into(c, body, bd, [&]() { enqueue_division_setup(c); });
    if (rc) return rc;
    cudaGraphConditionalHandle h_try = 0;
    CK(cudaGraphConditionalHandleCreate(&h_try, body, 1, cudaGraphCondAssignDefault));   // the first try always runs
    cudaGraph_t tries;
    rc = add_conditional(c, body, bd, h_try, cudaGraphCondTypeWhile, &tries);
    if (rc) return rc;
    std::vector<cudaGraphNode_t> tb;
    rc = capture_into(c, tries, tb, [&]() {
        launch_div_try_round(c->geom, c->phys, c->ctrl, c->dp, c->grid, c->bin_start, c->sorted_cell,
                             c->sorted_geom, c->div_flags, c->mothers, c->div_check, c->div_sat, c->d1, c->d2,
                             c->dlen, c->dgrowth, c->div_ok, h_try, c->st);
    });
    if (rc) return rc;
    return capture_into(c, body, bd, [&]() { enqueue_division_commit(c); enqueue_rebuild(c); });
}

// After the accepted step (simulation.hpp:1831-2022): basal-only compaction and its
// rebuild, the periodic neighbor rebuild, then switching, the ramps and local viscosity,
// which read the neighbor rows as they stand after those rebuilds.
static void enqueue_basal_test(abm_ctx* c, unsigned long long cond, int use_cond)
{
    launch_basal_flags(c->geom, c->ctrl, c->sw, c->keep, c->cap, c->st);
    launch_scan(c->keep, &c->ctrl->n, c->keep_rank, c->scan_sums, c->cap, c->st);
    launch_basal_decide(c->ctrl, c->keep, c->keep_rank, cond, use_cond, c->st);
}

static void enqueue_basal_compact(abm_ctx* c)
{
    launch_basal_compact(c->geom, c->vel, c->phys, c->geom_c, c->vel_c, c->phys_c, c->ctrl, c->keep, c->keep_rank,
                         c->cap, c->st, c->sp.fric ? c->feta : nullptr, c->staging);
}

static void enqueue_switch_cells(abm_ctx* c)
{
    if (c->sw.mode != 0) launch_switch_cells(c->geom, c->phys, c->ctrl, c->sw, c->cap, c->st);
    if (c->sw.modulate)
        launch_modulate_viscosity(c->geom, c->phys, c->ctrl, c->row_ptr, c->col, c->sw, c->cap, c->st);
}

// the same on a stream, the two rebuild decisions read back on the host
static int post_step_direct(abm_ctx* c)
{
    Ctrl h;
    if (c->sw.basal)
    {
        enqueue_basal_test(c, 0, 0);
        CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        if (h.n_keep < h.n) { enqueue_basal_compact(c); enqueue_rebuild(c); }
    }
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (!h.halted && h.iter % c->p.iter_update_neighbors == 0) enqueue_rebuild(c);
    enqueue_switch_cells(c);
    CK(cudaGetLastError());
    return ABM_OK;
}

// the same as graph nodes: IF(a cell is dropped){compaction + rebuild},
// IF(iteration counter % iter_update_neighbors == 0){rebuild}, then the switching kernels
static int append_post_step(abm_ctx* c, cudaGraph_t G, std::vector<cudaGraphNode_t>& deps)
{
    int rc;
    if (c->sw.basal)
    {
        cudaGraphConditionalHandle h_basal = 0;
        CK(cudaGraphConditionalHandleCreate(&h_basal, G, 0, cudaGraphCondAssignDefault));
        rc = capture_into(c, G, deps, [&]() { enqueue_basal_test(c, h_basal, 1); });
        if (rc) return rc;
        cudaGraph_t body;
        rc = add_conditional(c, G, deps, h_basal, cudaGraphCondTypeIf, &body);
        if (rc) return rc;
        std::vector<cudaGraphNode_t> bd;
        rc = capture_into(c, body, bd, [&]() { enqueue_basal_compact(c); enqueue_rebuild(c); });
        if (rc) return rc;
    }
    cudaGraphConditionalHandle h_reb = 0;
    CK(cudaGraphConditionalHandleCreate(&h_reb, G, 0, cudaGraphCondAssignDefault));
    rc = capture_into(c, G, deps, [&]() {
        launch_periodic_rebuild_cond(c->ctrl, c->p.iter_update_neighbors, h_reb, c->st);
    });
    if (rc) return rc;
    cudaGraph_t body;
    rc = add_conditional(c, G, deps, h_reb, cudaGraphCondTypeIf, &body);
    if (rc) return rc;
    std::vector<cudaGraphNode_t> bd;
    rc = capture_into(c, body, bd, [&]() { enqueue_rebuild(c); });
    if (rc) return rc;
    if (c->sw.mode != 0) return capture_into(c, G, deps, [&]() { enqueue_switch_cells(c); });
    return ABM_OK;
}

// One loop iteration as a graph with conditional nodes, appended to G after `deps`
// (empty: root nodes); `deps` becomes the iteration's leaf set:
//   [division count] -> IF(n_divide > 0){division + rebuild}
//   -> pair force -> [proposal] -> trial -> WHILE(retry requested){retry} -> final
// With the learned controller a passing proposal closes the step in the trial, and
// the rest runs only after a failed one:
//   ... -> trial -> IF(proposal failed){retry x max_tries (each exits at once when
//   no retry is pending) -> final}
static int append_iteration(abm_ctx* c, cudaGraph_t G, std::vector<cudaGraphNode_t>& deps)
{
    // every handle must belong to a conditional node of this graph, or instantiation fails
    cudaGraphConditionalHandle h_div = 0, h_retry = 0, h_run = 0;
    const bool branch = c->sp.propose != 0;
    const bool retries = c->p.max_tries_update_stepsize > 0 && !branch;
    if (retries) CK(cudaGraphConditionalHandleCreate(&h_retry, G, 0, cudaGraphCondAssignDefault));
    if (branch) CK(cudaGraphConditionalHandleCreate(&h_run, G, 0, cudaGraphCondAssignDefault));
    int rc;
    if (c->div_enabled)
    {
        CK(cudaGraphConditionalHandleCreate(&h_div, G, 0, cudaGraphCondAssignDefault));
        rc = capture_into(c, G, deps, [&]() { launch_div_count(c->phys, c->ctrl, c->dp, c->div_flags, h_div, 1, c->st); });
        if (rc) return rc;
        cudaGraph_t body;
        rc = add_conditional(c, G, deps, h_div, cudaGraphCondTypeIf, &body);
        if (rc) return rc;
        rc = capture_division_body(c, body);
        if (rc) return rc;
    }
    if (c->verlet)
    {
        rc = capture_into(c, G, deps, [&]() { enqueue_verlet_step(c); });
        if (rc) return rc;
        if (c->post_on)
        {
            rc = append_post_step(c, G, deps);
            if (rc) return rc;
        }
        if (c->frame_slots > 0) return capture_into(c, G, deps, [&]() { enqueue_frame_snapshot(c); });
        return ABM_OK;
    }
    PairGather pg = loop_gather(c);
    rc = capture_into(c, G, deps, [&]() {
        enqueue_loop_pair_force(c);
        enqueue_friction_rounds(c, MODE_TRIAL, pg);
        launch_attempt(MODE_TRIAL, c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->geom_c, c->vel_c, nullptr,
                       c->k0buf, 0.0, 0, c->cap, c->st, h_retry, (retries ? 1 : 0) | (branch ? 2 : 0), pg, c->dims,
                       h_run);
    });
    if (rc) return rc;
    auto retry_attempt = [&](int use_cond) {
        enqueue_friction_rounds(c, MODE_RETRY, pg);
        launch_attempt(MODE_RETRY, c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->geom_c, c->vel_c,
                       nullptr, c->k0buf, 0.0, 0, c->cap, c->st, h_retry, use_cond, pg, c->dims);
    };
    auto final_attempt = [&]() {
        enqueue_friction_rounds(c, MODE_FINAL, pg);
        launch_attempt(MODE_FINAL, c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->geom_c, c->vel_c, nullptr,
                       c->k0buf, 0.0, 0, c->cap, c->st, 0, 0, pg, c->dims);
    };
    if (branch)
    {
        cudaGraph_t body;
        rc = add_conditional(c, G, deps, h_run, cudaGraphCondTypeIf, &body);
        if (rc) return rc;
        std::vector<cudaGraphNode_t> bd;
        rc = capture_into(c, body, bd, [&]() {
            for (int r = 0; r < c->p.max_tries_update_stepsize; ++r) retry_attempt(0);
            final_attempt();
        });
        if (rc) return rc;
    }
    else
    {
        if (retries)
        {
            cudaGraph_t body;
            rc = add_conditional(c, G, deps, h_retry, cudaGraphCondTypeWhile, &body);
            if (rc) return rc;
            std::vector<cudaGraphNode_t> bd;
            rc = capture_into(c, body, bd, [&]() { retry_attempt(1); });
            if (rc) return rc;
        }
        rc = capture_into(c, G, deps, final_attempt);
        if (rc) return rc;
    }
    if (c->post_on)
    {
        rc = append_post_step(c, G, deps);
        if (rc) return rc;
    }
    // frames: the snapshot of a frame the accepted step marked
    if (c->frame_slots > 0) return capture_into(c, G, deps, [&]() { enqueue_frame_snapshot(c); });
    return ABM_OK;
}

static int instantiate_iterations(abm_ctx* c, int k, cudaGraphExec_t* exec)
{
    cudaGraph_t G;
    CK(cudaGraphCreate(&G, 0));
    std::vector<cudaGraphNode_t> deps;
    for (int r = 0; r < k; ++r)
    {
        int rc = append_iteration(c, G, deps);
        if (rc) { cudaGraphDestroy(G); return rc; }
    }
    cudaError_t inst = cudaGraphInstantiate(exec, G, 0);
    cudaGraphDestroy(G);
    CK(inst);
    return ABM_OK;
}

// One iteration per graph, and (for long loops) iter_k iterations per graph, iter_k
// the largest of 10, 5, 4, 2 that divides iter_update_neighbors, so that a K-graph
// launched at a multiple of iter_k never straddles a periodic rebuild.  The fixed
// cost of a graph launch (host submission, the conditional nodes' scheduling) is
// paid once per iter_k iterations.
static int build_iteration_graph(abm_ctx* c)
{
    int rc = instantiate_iterations(c, 1, &c->g_iter);
    if (rc) return rc;
    c->iter_k = 1;
    for (int k : {10, 5, 4, 2})
        if (c->p.iter_update_neighbors % k == 0) { c->iter_k = k; break; }
    if (c->iter_k > 1) return instantiate_iterations(c, c->iter_k, &c->g_iter_k);
    return ABM_OK;
}

// Division outside a graph: the flag count decides on the host whether the
// body and the neighbor rebuild run.
static int divide_now(abm_ctx* c, bool rebuild, int* n_divided)
{
    launch_div_count(c->phys, c->ctrl, c->dp, c->div_flags, 0, 0, c->st);
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (n_divided) *n_divided = h.n_divide;
    if (h.n_divide > 0)
    {
        enqueue_division_body(c);
        if (rebuild) enqueue_rebuild(c);
        else c->nbrs_valid = false;
        CK(cudaGetLastError());
    }
    return ABM_OK;
}

static int ready_for_forces(abm_ctx* c)
{
    if (!c->cells_loaded) return fail(c, ABM_ERR_STATE, "no cells uploaded");
    if (c->dims == 3 && c->p.adhesion_mode != 0 && c->jkr_n < 2) return fail(c, ABM_ERR_STATE, "JKR table not set");
    return ABM_OK;
}

int abm_build_neighbors(abm_ctx* c, int* m)
{
    if (!c) return ABM_ERR_ARG;
    if (!c->cells_loaded) return fail(c, ABM_ERR_STATE, "no cells uploaded");
    enqueue_rebuild(c);
    CK(cudaGetLastError());
    c->nbrs_valid = true;
    int rc = check_status(c);
    if (rc) return rc;
    if (m)
    {
        Ctrl h;
        CK(cudaMemcpy(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
        *m = h.n_dir / 2;
    }
    return ABM_OK;
}

int abm_download_neighbors(abm_ctx* c, double* rows, int ld, int cap, int* m)
{
    if (!c) return ABM_ERR_ARG;
    if (!c->nbrs_valid) return fail(c, ABM_ERR_STATE, "neighbors not built");
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int mm = h.n_dir / 2;
    if (m) *m = mm;
    if (!rows) return ABM_OK;
    if (cap < mm || ld < mm) return fail(c, ABM_ERR_CAPACITY, "row buffer too small");
    launch_count_lower(c->ctrl, c->row_ptr, c->col, c->nbr_count, c->cap, c->st);
    launch_scan(c->nbr_count, &c->ctrl->n, c->key, c->scan_sums, c->cap, c->st);
    const int ncol = c->dims == 2 ? 6 : 7;
    double* d_rows = nullptr;
    CK(cudaMallocAsync(&d_rows, (size_t)std::max(mm, 1) * ncol * sizeof(double), c->st));
    launch_table_rows(c->ctrl, c->row_ptr, c->col, c->key, c->geom, d_rows, std::max(mm, 1), c->cap, c->st, c->dims);
    if (mm > 0)
        CK(cudaMemcpy2DAsync(rows, (size_t)ld * sizeof(double), d_rows, (size_t)mm * sizeof(double),
                             (size_t)mm * sizeof(double), ncol, cudaMemcpyDeviceToHost, c->st));
    CK(cudaFreeAsync(d_rows, c->st));
    CK(cudaStreamSynchronize(c->st));
    return ABM_OK;
}

int abm_upload_neighbors(abm_ctx* c, const double* rows, int m, int ld)
{
    if (!c || (m > 0 && !rows) || ld < m) return ABM_ERR_ARG;
    if (!c->cells_loaded) return fail(c, ABM_ERR_STATE, "no cells uploaded");
    const int n = c->n_host;
    std::vector<std::vector<int>> adj(n);
    for (int k = 0; k < m; ++k)
    {
        int i = (int)rows[k], j = (int)rows[(size_t)ld + k];
        if (i < 0 || j < 0 || i >= n || j >= n || i == j) return fail(c, ABM_ERR_ARG, "bad neighbor row");
        adj[i].push_back(j); adj[j].push_back(i);
    }
    std::vector<int> rp(n + 1, 0), cl;
    for (int i = 0; i < n; ++i)
    {
        std::sort(adj[i].begin(), adj[i].end());
        if ((int)adj[i].size() > c->cap_nbr) return fail(c, ABM_ERR_CAPACITY, "neighbors per cell exceed capacity");
        rp[i + 1] = rp[i] + (int)adj[i].size();
        cl.insert(cl.end(), adj[i].begin(), adj[i].end());
    }
    CK(cudaMemcpyAsync(c->row_ptr, rp.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, c->st));
    if (!cl.empty()) CK(cudaMemcpyAsync(c->col, cl.data(), cl.size() * sizeof(int), cudaMemcpyHostToDevice, c->st));
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    h.n_dir = (int)cl.size();
    CK(cudaMemcpy(c->ctrl, &h, sizeof(Ctrl), cudaMemcpyHostToDevice));
    launch_csr_rev(c->ctrl, c->row_ptr, c->col, c->lower_end, c->rev, c->cap, c->st);
    launch_pair_list(c->ctrl, c->row_ptr, c->lower_end, c->col, c->rev, c->nbr_count, c->pair_start, c->scan_sums,
                     c->pairs, c->cap, c->st);
    if (c->dims == 2 && c->p.adhesion_mode != 0)
        launch_adhere_flags(c->ctrl, c->row_ptr, c->col, c->geom, c->p.R, c->p.Rcell, c->adhere, c->cap, c->st);
    CK(cudaGetLastError());
    c->nbrs_valid = true;
    return ABM_OK;
}

// ---------------------------------------------------------------------------
// Exact binary checkpoints. The reference resumes a run from its text frames, whose
// 10 significant digits move each value by up to 5e-10 of itself. A checkpoint keeps
// the FP64 bits of the cells, the neighbor set, the lineage, the clock and the state
// the controllers carry from one iteration to the next (the last HIST steps' dt,
// scaled errors and accept flags, the step statistics the proposal reads, the loop's
// counters). Everything else on the device is rebuilt or reset by the upload: the
// active pair list and the attempt order depend on nothing but the cells and the
// neighbor set, and they change no result bit. The random draws are keyed by the
// iteration, which the checkpoint restores. So a context created with the same
// parameters (and network weights), loaded from a checkpoint written at an
// iteration boundary, continues bit for bit where the uninterrupted run continues.
//
// File: "ABMCKP01", six int32 (dims, ncols, n, pairs m, lineage length, 0), the
// CkState block, cells (ncols x n doubles, column-major), pair cell indices (m int32
// i, then m int32 j, each pair once as the neighbor table lists it), lineage (int32).
// Host byte order.
struct CkState {
    double t, dt, dt_try, factor, last_max_error, last_trial_error, dt_prev;
    double hist_dt[HIST], hist_err[HIST];
    long long iter, since_div, hist_pos, first_passed, hist_acc[HIST];
    long long attempts, retries, iterations, rebuilds, divisions, div_events, rejected, cell_steps,
        basal_dropped, last_div_tries;
    unsigned long long st_vmax_bits, st_ovl_bits[2], st_v2_fx, st_g_fx, st_near_div;
};
static_assert(sizeof(CkState) % 8 == 0, "checkpoint state block is made of 8-byte fields");
static const char CK_MAGIC[8] = {'A', 'B', 'M', 'C', 'K', 'P', '0', '1'};

static void ck_from_ctrl(const Ctrl& h, CkState& s)
{
    s.t = h.t; s.dt = h.dt; s.dt_try = h.dt_try; s.factor = h.factor;
    s.last_max_error = h.last_max_error; s.last_trial_error = h.last_trial_error; s.dt_prev = h.dt_prev;
    for (int k = 0; k < HIST; ++k)
    {
        s.hist_dt[k] = h.hist_dt[k]; s.hist_err[k] = h.hist_err[k]; s.hist_acc[k] = h.hist_acc[k];
    }
    s.iter = h.iter; s.since_div = h.since_div; s.hist_pos = h.hist_pos; s.first_passed = h.first_passed;
    s.attempts = h.attempts; s.retries = h.retries; s.iterations = h.iterations; s.rebuilds = h.rebuilds;
    s.divisions = h.divisions; s.div_events = h.div_events; s.rejected = h.rejected;
    s.cell_steps = h.cell_steps; s.basal_dropped = h.basal_dropped; s.last_div_tries = h.last_div_tries;
    s.st_vmax_bits = h.st_vmax_bits; s.st_ovl_bits[0] = h.st_ovl_bits[0]; s.st_ovl_bits[1] = h.st_ovl_bits[1];
    s.st_v2_fx = h.st_v2_fx; s.st_g_fx = h.st_g_fx; s.st_near_div = h.st_near_div;
}

static void ck_to_ctrl(const CkState& s, Ctrl& h)
{
    h.t = s.t; h.dt = s.dt; h.dt_try = s.dt_try; h.factor = s.factor;
    h.last_max_error = s.last_max_error; h.last_trial_error = s.last_trial_error; h.dt_prev = s.dt_prev;
    for (int k = 0; k < HIST; ++k)
    {
        h.hist_dt[k] = s.hist_dt[k]; h.hist_err[k] = s.hist_err[k]; h.hist_acc[k] = (int)s.hist_acc[k];
    }
    h.iter = (int)s.iter; h.since_div = (int)s.since_div; h.hist_pos = (int)s.hist_pos;
    h.first_passed = (int)s.first_passed;
    h.attempts = s.attempts; h.retries = s.retries; h.iterations = s.iterations; h.rebuilds = s.rebuilds;
    h.divisions = s.divisions; h.div_events = s.div_events; h.rejected = s.rejected;
    h.cell_steps = s.cell_steps; h.basal_dropped = s.basal_dropped; h.last_div_tries = (int)s.last_div_tries;
    h.st_vmax_bits = s.st_vmax_bits; h.st_ovl_bits[0] = s.st_ovl_bits[0]; h.st_ovl_bits[1] = s.st_ovl_bits[1];
    h.st_v2_fx = s.st_v2_fx; h.st_g_fx = s.st_g_fx; h.st_near_div = s.st_near_div;
}

int abm_save_checkpoint(abm_ctx* c, const char* path)
{
    if (!c || !path) return ABM_ERR_ARG;
    if (!c->cells_loaded) return fail(c, ABM_ERR_STATE, "no cells uploaded");
    if (!c->nbrs_valid) return fail(c, ABM_ERR_STATE, "neighbors not built");
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const int n = h.n, ncols = c->ncols, n_par = h.n_parents;
    std::vector<double> cells((size_t)std::max(n, 1) * ncols);
    int rc = abm_download_cells(c, cells.data(), std::max(n, 1));
    if (rc) return rc;
    int m = 0;
    rc = abm_download_neighbors(c, nullptr, 0, 0, &m);
    if (rc) return rc;
    const int tcols = c->dims == 2 ? 6 : 7;
    std::vector<double> rows((size_t)std::max(m, 1) * tcols);
    if (m > 0 && (rc = abm_download_neighbors(c, rows.data(), m, m, &m))) return rc;
    std::vector<int> pairs((size_t)2 * m);
    for (int k = 0; k < m; ++k) { pairs[k] = (int)rows[k]; pairs[(size_t)m + k] = (int)rows[(size_t)m + k]; }
    std::vector<int> parents((size_t)std::max(n_par, 0));
    if (n_par > 0 && (rc = abm_get_parents(c, parents.data(), n_par, nullptr))) return rc;
    CkState s;
    std::memset(&s, 0, sizeof(s));
    ck_from_ctrl(h, s);
    const int hdr[6] = {c->dims, ncols, n, m, n_par, 0};
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(c, ABM_ERR_ARG, std::string("cannot open ") + path + " for writing");
    bool ok = std::fwrite(CK_MAGIC, 1, 8, f) == 8 && std::fwrite(hdr, sizeof(int), 6, f) == 6 &&
              std::fwrite(&s, sizeof(s), 1, f) == 1;
    if (ok && n > 0) ok = std::fwrite(cells.data(), sizeof(double), (size_t)n * ncols, f) == (size_t)n * ncols;
    if (ok && m > 0) ok = std::fwrite(pairs.data(), sizeof(int), pairs.size(), f) == pairs.size();
    if (ok && n_par > 0) ok = std::fwrite(parents.data(), sizeof(int), parents.size(), f) == parents.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(c, ABM_ERR_ARG, std::string("write failed: ") + path);
    return ABM_OK;
}

int abm_load_checkpoint(abm_ctx* c, const char* path)
{
    if (!c || !path) return ABM_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(c, ABM_ERR_ARG, std::string("cannot open ") + path);
    char magic[8];
    int hdr[6];
    CkState s;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, CK_MAGIC, 8) == 0 &&
              std::fread(hdr, sizeof(int), 6, f) == 6 && std::fread(&s, sizeof(s), 1, f) == 1;
    const int dims = ok ? hdr[0] : 0, ncols = ok ? hdr[1] : 0, n = ok ? hdr[2] : -1, m = ok ? hdr[3] : -1,
              n_par = ok ? hdr[4] : -1;
    if (!ok || n < 0 || m < 0 || n_par < 0 || ncols <= 0 || ncols > STAGING_COLS)
    {
        std::fclose(f);
        return fail(c, ABM_ERR_ARG, std::string("not a checkpoint of this library: ") + path);
    }
    if (dims != c->dims)
    {
        std::fclose(f);
        return fail(c, ABM_ERR_ARG, "the checkpoint belongs to the other model (2-D / 3-D)");
    }
    if (n > c->cap)
    {
        std::fclose(f);
        return fail(c, ABM_ERR_CAPACITY, "the checkpoint holds more cells than cap_cells");
    }
    std::vector<double> cells((size_t)std::max(n, 1) * ncols);
    std::vector<int> pairs((size_t)2 * m), parents((size_t)n_par);
    if (n > 0) ok = std::fread(cells.data(), sizeof(double), (size_t)n * ncols, f) == (size_t)n * ncols;
    if (ok && m > 0) ok = std::fread(pairs.data(), sizeof(int), pairs.size(), f) == pairs.size();
    if (ok && n_par > 0) ok = std::fread(parents.data(), sizeof(int), parents.size(), f) == parents.size();
    if (ok) ok = std::fgetc(f) == EOF;                // nothing after the lineage
    std::fclose(f);
    if (!ok) return fail(c, ABM_ERR_ARG, std::string("truncated or oversized checkpoint: ") + path);
    if (!(s.dt > 0) || s.iter < 0 || s.iter > INT_MAX || s.hist_pos < 0 || s.hist_pos >= HIST)
        return fail(c, ABM_ERR_ARG, "the checkpoint's clock or controller history is out of range");
    // the checks abm_upload_neighbors makes, before anything reaches the context, so
    // that a rejected file leaves it as it was
    std::vector<int> degree((size_t)std::max(n, 1), 0);
    for (int k = 0; k < m; ++k)
    {
        const int i = pairs[k], j = pairs[(size_t)m + k];
        if (i < 0 || j < 0 || i >= n || j >= n || i == j)
            return fail(c, ABM_ERR_ARG, "the checkpoint's neighbor set names a cell it does not hold");
        if (++degree[i] > c->cap_nbr || ++degree[j] > c->cap_nbr)
            return fail(c, ABM_ERR_CAPACITY, "the checkpoint's neighbors per cell exceed cap_neighbors_per_cell");
    }
    int rc = abm_upload_cells(c, cells.data(), n, ncols, std::max(n, 1));
    if (rc) return rc;
    if ((rc = abm_set_parents(c, n_par > 0 ? parents.data() : nullptr, n_par))) return rc;
    std::vector<double> rows((size_t)std::max(m, 1) * 2);
    for (int k = 0; k < m; ++k) { rows[k] = pairs[k]; rows[(size_t)m + k] = pairs[(size_t)m + k]; }
    if ((rc = abm_upload_neighbors(c, rows.data(), m, std::max(m, 1)))) return rc;
    if ((rc = abm_set_clock(c, s.t, s.dt, (int)s.iter))) return rc;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    ck_to_ctrl(s, h);
    CK(cudaMemcpy(c->ctrl, &h, sizeof(Ctrl), cudaMemcpyHostToDevice));
    return ABM_OK;
}

// n x 6 (3-D) or the (x, y, nx, ny) columns n x 4 (2-D)
static int download_gen6(abm_ctx* c, const Gen6* src, double* out)
{
    int n = c->n_host;
    if (n == 0) return ABM_OK;
    launch_gen6_to_colmajor(src, n, c->staging, c->st);
    if (c->dims == 2)
    {
        const int cols[4] = {0, 1, 3, 4};
        for (int k = 0; k < 4; ++k)
            CK(cudaMemcpyAsync(out + (size_t)k * n, c->staging + (size_t)cols[k] * n, (size_t)n * sizeof(double),
                               cudaMemcpyDeviceToHost, c->st));
    }
    else
        CK(cudaMemcpyAsync(out, c->staging, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return ABM_OK;
}

int abm_cell_cell_forces(abm_ctx* c, double* out)
{
    if (!c || !out) return ABM_ERR_ARG;
    int rc = ready_for_forces(c);
    if (rc) return rc;
    if (!c->nbrs_valid) return fail(c, ABM_ERR_STATE, "neighbors not built");
    enqueue_pair_force(c, 1);
    CK(cudaGetLastError());
    if (c->dims == 2)
    {
        // the reference's 2-D dE/dq projects each pair's torque with the current n
        const int n = c->n_host;
        if (n == 0) return ABM_OK;
        launch_pair_dEdq_2d(c->geom, c->fcc, c->ctrl, c->staging, c->cap, c->st);
        CK(cudaMemcpyAsync(out, c->staging, (size_t)n * 4 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        return ABM_OK;
    }
    return download_gen6(c, c->fcc, out);
}

int abm_get_velocities(abm_ctx* c, double* out)
{
    if (!c || !out) return ABM_ERR_ARG;
    int rc = ready_for_forces(c);
    if (rc) return rc;
    if (!c->nbrs_valid) return fail(c, ABM_ERR_STATE, "neighbors not built");
    enqueue_pair_force(c, 1);
    launch_velocities(c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->gen_tmp, c->cap, c->st, c->dims);
    CK(cudaGetLastError());
    rc = download_gen6(c, c->gen_tmp, out);
    if (rc) return rc;
    return check_status(c);
}

__global__ void k_clear_eval(Ctrl* c) { c->eval_err_bits = 0ull; }

int abm_rk_attempt(abm_ctx* c, double dt, int attempt, double* cells_out, double* errors_out,
                   double* max_scaled_error)
{
    if (!c || !(dt > 0)) return ABM_ERR_ARG;
    if (c->verlet) return fail(c, ABM_ERR_STATE, "the context integrates with velocity Verlet (no RK attempt)");
    int rc = ready_for_forces(c);
    if (rc) return rc;
    if (!c->nbrs_valid) return fail(c, ABM_ERR_STATE, "neighbors not built");
    enqueue_pair_force(c, 1);
    k_clear_eval<<<1, 1, 0, c->st>>>(c->ctrl);
    PairGather pg = {0, c->row_ptr, c->lower_end, c->jbuf, nullptr, c->fbuf, c->fmask, c->ystage, c->cap};
    enqueue_friction_rounds(c, 3, pg, dt, attempt);
    launch_attempt(3, c->geom, c->vel, c->phys, c->fcc, c->ctrl, c->sp, c->geom_c, c->vel_c, c->gen_tmp,
                   c->k0buf, dt, attempt, c->cap, c->st, 0, 0, pg, c->dims);
    CK(cudaGetLastError());
    const int n = c->n_host;
    if (cells_out && n > 0)
    {
        if (c->dims == 2) launch_cells_to_colmajor_2d(c->geom_c, c->vel_c, c->phys, n, c->ncols, n, c->staging, c->st);
        else launch_cells_to_colmajor(c->geom_c, c->vel_c, c->phys, n, c->ncols, n, c->has_gamma, c->staging, c->st);
        rc = stage_eta_column(c, c->feta, n);
        if (rc) return rc;
        CK(cudaMemcpyAsync(cells_out, c->staging, (size_t)n * c->ncols * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    }
    if (errors_out)
    {
        rc = download_gen6(c, c->gen_tmp, errors_out);
        if (rc) return rc;
    }
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (max_scaled_error)
    {
        double e;
        memcpy(&e, &h.eval_err_bits, sizeof(double));
        *max_scaled_error = std::max(e, c->p.min_error);
    }
    return check_status(c);
}

int abm_grow(abm_ctx* c, double dt)
{
    if (!c) return ABM_ERR_ARG;
    if (!c->cells_loaded) return fail(c, ABM_ERR_STATE, "no cells uploaded");
    launch_grow(c->geom, c->phys, c->ctrl, c->p.R, dt, c->cap, c->st);
    k_screen_stale<<<1, 1, 0, c->st>>>(c->ctrl);
    CK(cudaGetLastError());
    return ABM_OK;
}

int abm_divide(abm_ctx* c, int* n_divided)
{
    if (!c) return ABM_ERR_ARG;
    if (!c->cells_loaded) return fail(c, ABM_ERR_STATE, "no cells uploaded");
    int rc = divide_now(c, false, n_divided);
    if (rc) return rc;
    rc = check_status(c);
    Ctrl h;
    CK(cudaMemcpy(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    c->n_host = h.n;
    return rc;
}

const char* abm_graph_info(const abm_ctx* c)
{
    if (!c) return "";
    if (!c->g_iter) return "no iteration graph yet";
    return c->graph_fallback ? c->graph_note.c_str() : "conditional";
}

int abm_last_division_tries(abm_ctx* c, int* tries)
{
    if (!c || !tries) return ABM_ERR_ARG;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *tries = h.last_div_tries;
    return ABM_OK;
}

int abm_get_stats(abm_ctx* c, abm_stats* s)
{
    if (!c || !s) return ABM_ERR_ARG;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    s->iterations = h.iterations; s->attempts = h.attempts; s->retries = h.retries;
    s->rebuilds = h.rebuilds; s->divisions = h.divisions;
    s->t = h.t; s->dt = h.dt; s->last_max_error = h.last_max_error;
    s->n_cells = h.n; s->n_pairs = h.n_dir / 2;
    s->rejected = h.rejected; s->log_rows = h.log_rows; s->cell_steps = h.cell_steps;
    return check_status(c);
}

int abm_iterate(abm_ctx* c, int n_iters, int n_cells_stop, abm_stats* stats)
{
    if (!c || n_iters < 0) return ABM_ERR_ARG;
    int rc = ready_for_forces(c);
    if (rc) return rc;
    if (c->sp.network && !c->mlp_loaded)
        return fail(c, ABM_ERR_STATE, "the learned controller needs weights (abm_stepsize_set_weights)");
    if (!c->nbrs_valid)
    {
        enqueue_rebuild(c);
        c->nbrs_valid = true;
    }
    if (c->p.use_graphs)
    {
        if (!c->g_iter && !c->graph_fallback)
        {
            rc = build_iteration_graph(c);
            if (rc)
            {
                // conditional nodes unavailable: keep the error for abm_graph_info and fall back to
                // a straight-line graph (retries exit early) with division decided on the host
                c->graph_note = c->err;
                c->graph_fallback = true;
                cudaGetLastError();
                drop_iteration_graphs(c);
            }
        }
        if (c->graph_fallback && !c->g_iter) { rc = capture(c, enqueue_iteration, &c->g_iter); if (rc) return rc; }
        if (!c->g_rebuild) { rc = capture(c, enqueue_rebuild, &c->g_rebuild); if (rc) return rc; }
    }
    for (int k = 0, next_check = 0; k < n_iters;)
    {
        if (n_cells_stop > 0 && c->div_enabled && k >= next_check)
        {
            Ctrl h;
            CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
            if (h.n >= n_cells_stop) break;
            next_check = k + 16;
        }
        int step = 1;
        if (c->p.use_graphs && !c->graph_fallback)
        {
            if (c->g_iter_k && c->host_iter % c->iter_k == 0 && n_iters - k >= c->iter_k)
            {
                CK(cudaGraphLaunch(c->g_iter_k, c->st));
                step = c->iter_k;
            }
            else CK(cudaGraphLaunch(c->g_iter, c->st));
        }
        else
        {
            if (c->div_enabled) { rc = divide_now(c, true, nullptr); if (rc) return rc; }
            if (c->post_on)
            {
                if (c->verlet) enqueue_verlet_step(c);
                else
                {
                    enqueue_loop_pair_force(c);
                    enqueue_attempts(c);
                }
                rc = post_step_direct(c);
                if (rc) return rc;
                if (c->frame_slots > 0) enqueue_frame_snapshot(c);
            }
            else if (c->p.use_graphs) CK(cudaGraphLaunch(c->g_iter, c->st));
            else enqueue_iteration(c);
        }
        c->host_iter += step;
        k += step;
        // with the post-step kernels on, the periodic rebuild is part of the iteration
        if (!c->post_on && c->host_iter % c->p.iter_update_neighbors == 0)
        {
            if (c->p.use_graphs) CK(cudaGraphLaunch(c->g_rebuild, c->st));
            else enqueue_rebuild(c);
        }
    }
    CK(cudaGetLastError());
    if (stats) return abm_get_stats(c, stats);
    return ABM_OK;
}

int abm_profile_iterations(abm_ctx* c, int n_iters, abm_profile* prof)
{
    if (!c || !prof || n_iters < 0) return ABM_ERR_ARG;
    if (c->post_on) return fail(c, ABM_ERR_STATE, "the profile covers the loop without switching or basal-only compaction");
    if (c->verlet) return fail(c, ABM_ERR_STATE, "the profile covers the Runge-Kutta loop");
    int rc = ready_for_forces(c);
    if (rc) return rc;
    if (c->sp.network && !c->mlp_loaded)
        return fail(c, ABM_ERR_STATE, "the learned controller needs weights (abm_stepsize_set_weights)");
    if (!c->nbrs_valid) { enqueue_rebuild(c); c->nbrs_valid = true; }
    memset(prof, 0, sizeof(*prof));
    std::vector<cudaEvent_t> ev((size_t)n_iters * 4);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    std::vector<int> rebuilt(n_iters, 0);
    cudaStream_t st = c->st;
    for (int k = 0; k < n_iters; ++k)
    {
        cudaEvent_t* e = &ev[(size_t)k * 4];
        CK(cudaEventRecord(e[0], st));
        enqueue_loop_pair_force(c);
        CK(cudaEventRecord(e[1], st));
        enqueue_attempts(c);
        CK(cudaEventRecord(e[2], st));
        c->host_iter += 1;
        if (c->host_iter % c->p.iter_update_neighbors == 0) { enqueue_rebuild(c); rebuilt[k] = 1; }
        CK(cudaEventRecord(e[3], st));
    }
    CK(cudaStreamSynchronize(st));
    for (int k = 0; k < n_iters; ++k)
    {
        cudaEvent_t* e = &ev[(size_t)k * 4];
        float a, b, d;
        CK(cudaEventElapsedTime(&a, e[0], e[1]));
        CK(cudaEventElapsedTime(&b, e[1], e[2]));
        CK(cudaEventElapsedTime(&d, e[2], e[3]));
        prof->pair_force_ms += a;
        prof->attempt_ms += b;
        prof->pair_force_launches += 1;
        prof->attempt_launches += 2 + c->p.max_tries_update_stepsize;
        if (rebuilt[k]) { prof->rebuild_ms += d; prof->rebuild_launches += 1; }
    }
    prof->iterations = n_iters;
    for (auto& e : ev) cudaEventDestroy(e);
    return check_status(c);
}

// lower CSR entry of every neighbor row (i ascending, j < i ascending), on the host
static int row_entries(abm_ctx* c, std::vector<int>& entries)
{
    const int n = c->n_host;
    std::vector<int> rp(n + 1), cl;
    CK(cudaMemcpyAsync(rp.data(), c->row_ptr, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    cl.resize(rp[n]);
    if (rp[n] > 0) CK(cudaMemcpy(cl.data(), c->col, rp[n] * sizeof(int), cudaMemcpyDeviceToHost));
    entries.clear();
    for (int i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (cl[k] < i) entries.push_back(k);
    return ABM_OK;
}

int abm_get_adhesion_flags(abm_ctx* c, int* flags, int cap, int* m)
{
    if (!c || !m) return ABM_ERR_ARG;
    if (c->dims != 2) return fail(c, ABM_ERR_STATE, "adhesion flags belong to the 2-D model");
    if (!c->nbrs_valid) return fail(c, ABM_ERR_STATE, "neighbors not built");
    std::vector<int> e;
    int rc = row_entries(c, e);
    if (rc) return rc;
    *m = (int)e.size();
    if (!flags) return ABM_OK;
    if (cap < (int)e.size()) return fail(c, ABM_ERR_CAPACITY, "flag buffer too small");
    std::vector<unsigned char> a(std::max<size_t>(1, (size_t)c->cap * c->cap_nbr));
    if (!e.empty()) CK(cudaMemcpy(a.data(), c->adhere, (size_t)(e.back() + 1), cudaMemcpyDeviceToHost));
    for (size_t r = 0; r < e.size(); ++r) flags[r] = a[e[r]];
    return ABM_OK;
}

int abm_set_adhesion_flags(abm_ctx* c, const int* flags, int m)
{
    if (!c || (m > 0 && !flags)) return ABM_ERR_ARG;
    if (c->dims != 2) return fail(c, ABM_ERR_STATE, "adhesion flags belong to the 2-D model");
    if (!c->nbrs_valid) return fail(c, ABM_ERR_STATE, "neighbors not built");
    std::vector<int> e;
    int rc = row_entries(c, e);
    if (rc) return rc;
    if ((int)e.size() != m) return fail(c, ABM_ERR_ARG, "one flag per neighbor row");
    if (m == 0) return ABM_OK;
    std::vector<unsigned char> a((size_t)e.back() + 1, 0);
    for (int r = 0; r < m; ++r) a[e[r]] = flags[r] ? 1 : 0;
    CK(cudaMemcpy(c->adhere, a.data(), a.size(), cudaMemcpyHostToDevice));
    return ABM_OK;
}

int abm_set_cell_limit(abm_ctx* c, int n_max)
{
    if (!c || n_max < 0) return ABM_ERR_ARG;
    k_set_halt<<<1, 1, 0, c->st>>>(c->ctrl, n_max);
    CK(cudaGetLastError());
    return ABM_OK;
}

int abm_stepsize_set_weights(abm_ctx* c, const float* w, int n)
{
    if (!c || !w || n != MLP_NPARAM) return fail(c, ABM_ERR_ARG, "weights must have ABM_MLP_NPARAM entries");
    CK(cudaMemcpyAsync(c->mlp_w, w, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->mlp_loaded = true;
    return ABM_OK;
}

int abm_stepsize_get_weights(abm_ctx* c, float* w, int n)
{
    if (!c || !w || n != MLP_NPARAM) return fail(c, ABM_ERR_ARG, "weights must have ABM_MLP_NPARAM entries");
    CK(cudaMemcpyAsync(w, c->mlp_w, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return ABM_OK;
}

int abm_stepsize_get_log(abm_ctx* c, float* rows, int cap_rows, int* n_rows)
{
    if (!c || !n_rows || cap_rows < 0 || (cap_rows > 0 && !rows)) return fail(c, ABM_ERR_ARG, "bad arguments");
    *n_rows = 0;
    if (c->sp.log_cap <= 0) return ABM_OK;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const long long total = h.log_rows;
    const int cap = c->sp.log_cap;
    const int have = (int)std::min<long long>(total, cap);
    const int take = std::min(have, cap_rows);
    // oldest first: ring positions (total - have) .. total - 1, the first `take` of them
    std::vector<float> all((size_t)cap * MLP_LOG_COLS);
    CK(cudaMemcpy(all.data(), c->log_buf, all.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (int r = 0; r < take; ++r)
    {
        const long long pos = (total - have + r) % cap;
        memcpy(rows + (size_t)r * MLP_LOG_COLS, all.data() + (size_t)pos * MLP_LOG_COLS, MLP_LOG_COLS * sizeof(float));
    }
    *n_rows = take;
    return ABM_OK;
}

int abm_stepsize_clear_log(abm_ctx* c)
{
    if (!c) return ABM_ERR_ARG;
    Ctrl h;
    CK(cudaMemcpyAsync(&h, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    h.log_rows = 0;
    CK(cudaMemcpyAsync(c->ctrl, &h, sizeof(Ctrl), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return ABM_OK;
}

}   // extern "C"

// ---------------------------------------------------------------------------
// Batches of contexts (independent replicate biofilms) advanced by one graph
// ---------------------------------------------------------------------------
struct abm_batch {
    std::vector<abm_ctx*> ctxs;
    cudaStream_t st = nullptr;
    cudaGraphExec_t g_iter = nullptr, g_rebuild = nullptr;
    int k_rebuild = 100;
    std::vector<cudaEvent_t> ev;
    cudaEvent_t done = nullptr;
    std::string err;
};

namespace {
thread_local std::string g_batch_err;

int batch_fail(abm_batch* b, int code, const std::string& msg)
{
    if (b) b->err = msg;
    g_batch_err = msg;
    return code;
}

#define BK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    return batch_fail(b, ABM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

void batch_free(abm_batch* b)
{
    if (b->g_iter) cudaGraphExecDestroy(b->g_iter);
    if (b->g_rebuild) cudaGraphExecDestroy(b->g_rebuild);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    if (b->done) cudaEventDestroy(b->done);
    if (b->st) cudaStreamDestroy(b->st);
}
}   // namespace

extern "C" {

const char* abm_batch_last_error(void) { return g_batch_err.c_str(); }

int abm_batch_create(abm_ctx* const* ctxs, int n, abm_batch** out)
{
    g_batch_err.clear();
    if (!ctxs || n <= 0 || !out) return batch_fail(nullptr, ABM_ERR_ARG, "bad arguments");
    *out = nullptr;
    abm_batch* b = new abm_batch();
    b->ctxs.assign(ctxs, ctxs + n);
    b->k_rebuild = ctxs[0]->p.iter_update_neighbors;
    int dev = ctxs[0]->dev;
    for (abm_ctx* c : b->ctxs)
    {
        if (!c || !c->cells_loaded) { delete b; return batch_fail(nullptr, ABM_ERR_STATE, "every context needs cells"); }
        if (c->post_on)
        { delete b; return batch_fail(nullptr, ABM_ERR_STATE, "switching and basal-only contexts run through abm_iterate"); }
        if (c->dev != dev) { delete b; return batch_fail(nullptr, ABM_ERR_ARG, "contexts on different devices"); }
        if (c->p.iter_update_neighbors != b->k_rebuild)
        { delete b; return batch_fail(nullptr, ABM_ERR_ARG, "contexts must share iter_update_neighbors"); }
        if (c->sp.network && !c->mlp_loaded)
        { delete b; return batch_fail(nullptr, ABM_ERR_STATE, "a learned controller needs weights"); }
        if (c->dims == 3 && c->p.adhesion_mode != 0 && c->jkr_n < 2)
        { delete b; return batch_fail(nullptr, ABM_ERR_STATE, "JKR table not set"); }
        if (c->host_iter % b->k_rebuild != ctxs[0]->host_iter % b->k_rebuild)
        { delete b; return batch_fail(nullptr, ABM_ERR_STATE, "contexts must be in phase of the rebuild cadence"); }
        if (!c->nbrs_valid) { enqueue_rebuild(c); c->nbrs_valid = true; }
    }
    int rc = ABM_OK;
    cudaGraph_t G = nullptr, GR = nullptr;
    do {
        if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess)
        { rc = batch_fail(b, ABM_ERR_CUDA, "stream or event creation failed"); break; }
        b->ev.resize(n);
        for (int k = 0; k < n && !rc; ++k)
            if (cudaEventCreateWithFlags(&b->ev[k], cudaEventDisableTiming) != cudaSuccess)
                rc = batch_fail(b, ABM_ERR_CUDA, "event creation failed");
        if (rc) break;
        // one graph: every context's iteration as an independent branch
        if (cudaGraphCreate(&G, 0) != cudaSuccess || cudaGraphCreate(&GR, 0) != cudaSuccess)
        { rc = batch_fail(b, ABM_ERR_CUDA, "graph creation failed"); break; }
        for (abm_ctx* c : b->ctxs)
        {
            std::vector<cudaGraphNode_t> deps;
            rc = append_iteration(c, G, deps);
            if (rc) { rc = batch_fail(b, rc, "iteration graph of a context: " + c->err); break; }
            std::vector<cudaGraphNode_t> rdeps;
            rc = capture_into(c, GR, rdeps, [&]() { enqueue_rebuild(c); });
            if (rc) { rc = batch_fail(b, rc, "rebuild graph of a context: " + c->err); break; }
        }
        if (rc) break;
        if (cudaGraphInstantiate(&b->g_iter, G, 0) != cudaSuccess ||
            cudaGraphInstantiate(&b->g_rebuild, GR, 0) != cudaSuccess)
        { rc = batch_fail(b, ABM_ERR_CUDA, "graph instantiation failed"); break; }
    } while (0);
    if (G) cudaGraphDestroy(G);
    if (GR) cudaGraphDestroy(GR);
    if (rc) { batch_free(b); delete b; return rc; }
    *out = b;
    return ABM_OK;
}

// n_iters iterations of every context: one graph launch per iteration, the joint
// neighbor rebuild every iter_update_neighbors iterations (all contexts take their
// steps in lockstep, so their cadences coincide).  Work already queued on the
// contexts' streams runs first; their streams wait for the batch at the end.
int abm_batch_iterate(abm_batch* b, int n_iters)
{
    if (!b || n_iters < 0) return batch_fail(b, ABM_ERR_ARG, "bad arguments");
    const int n = (int)b->ctxs.size();
    for (int k = 0; k < n; ++k)
    {
        BK(cudaEventRecord(b->ev[k], b->ctxs[k]->st));
        BK(cudaStreamWaitEvent(b->st, b->ev[k], 0));
    }
    for (int it = 0; it < n_iters; ++it)
    {
        BK(cudaGraphLaunch(b->g_iter, b->st));
        bool rebuild = false;
        for (abm_ctx* c : b->ctxs)
        {
            c->host_iter += 1;
            rebuild = (c->host_iter % b->k_rebuild == 0);
        }
        if (rebuild) BK(cudaGraphLaunch(b->g_rebuild, b->st));
    }
    BK(cudaEventRecord(b->done, b->st));
    for (abm_ctx* c : b->ctxs) BK(cudaStreamWaitEvent(c->st, b->done, 0));
    BK(cudaGetLastError());
    return ABM_OK;
}

int abm_batch_synchronize(abm_batch* b)
{
    if (!b) return ABM_ERR_ARG;
    BK(cudaStreamSynchronize(b->st));
    for (abm_ctx* c : b->ctxs)
    {
        int rc = check_status(c);
        if (rc) return batch_fail(b, rc, c->err);
    }
    return ABM_OK;
}

int abm_batch_get_stream(abm_batch* b, void** stream)
{
    if (!b || !stream) return ABM_ERR_ARG;
    *stream = (void*)b->st;
    return ABM_OK;
}

int abm_batch_destroy(abm_batch* b)
{
    if (!b) return ABM_ERR_ARG;
    cudaStreamSynchronize(b->st);
    batch_free(b);
    delete b;
    return ABM_OK;
}

// ---------------------------------------------------------------------------
// Autotuner of the screened pair pass: tile of CSR entries per block and grid
// blocks per SM, timed on a scratch context holding the caller's state; the
// fastest candidate by CUDA events over `launches` launches wins.  No reference
// counterpart.
// ---------------------------------------------------------------------------
int abm_autotune_pair_tile(const abm_params* p, const double* cells, int n, int ncols, int ld,
                           const double* jkr_delta, const double* jkr_radius, int jkr_n, int launches,
                           int* best_tile, int* best_bpsm, float* ms_per_launch)
{
    g_batch_err.clear();
    if (!p || !cells || n <= 0 || !best_tile || !best_bpsm || launches <= 0)
        return batch_fail(nullptr, ABM_ERR_ARG, "bad arguments");
    abm_params q = *p;
    q.cap_cells = std::max(q.cap_cells, n);
    q.controller = ABM_CONTROLLER_REFERENCE;
    q.stepsize_log_capacity = 0;
    abm_ctx* c = nullptr;
    int rc = abm_create(&q, &c);
    if (rc == ABM_OK && q.adhesion_mode != 0 && (q.dims == 0 || q.dims == 3))
        rc = abm_set_jkr_table(c, jkr_delta, jkr_radius, jkr_n);
    if (rc == ABM_OK) rc = abm_upload_cells(c, cells, n, ncols, ld);
    int m = 0;
    if (rc == ABM_OK) rc = abm_build_neighbors(c, &m);
    const int tiles[3] = {512, 1024, 2048}, grids[3] = {1, 2, 4};
    float best = 0;
    *best_tile = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == ABM_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) rc = ABM_ERR_CUDA;
    for (int a = 0; a < 3 && rc == ABM_OK; ++a)
        for (int b = 0; b < 3 && rc == ABM_OK; ++b)
        {
            c->p.pair_tile = tiles[a];
            c->p.pair_blocks_per_sm = grids[b];
            enqueue_pair_force(c, 0);                       // warm-up
            cudaEventRecord(e0, c->st);
            for (int r = 0; r < launches; ++r) enqueue_pair_force(c, 0);
            cudaEventRecord(e1, c->st);
            float ms = 0;
            if (cudaEventSynchronize(e1) != cudaSuccess) { rc = ABM_ERR_CUDA; break; }
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= launches;
            if (ms_per_launch) ms_per_launch[3 * a + b] = ms;
            if (*best_tile == 0 || ms < best) { best = ms; *best_tile = tiles[a]; *best_bpsm = grids[b]; }
        }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    std::string why = c ? c->err : std::string("abm_create failed");
    if (c) abm_destroy(c);
    if (rc) return batch_fail(nullptr, rc, "autotune: " + why);
    return ABM_OK;
}

}   // extern "C"
