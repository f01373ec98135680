/*
 * C ABI of the B200 mechanics step for the kmnam/biofilm-ABMs 3-D model.
 *
 * The reference exposes no plugin or FFI layer: its seam is the set of
 * templated free functions that ABM-3d/ABM-3d-cpp/include/simulation.hpp's
 * runSimulation loop calls.  Each entry point below names the reference
 * function (file:line) it stands in for.  Arrays cross this boundary in the
 * reference's own layout: column-major double arrays (Eigen::Array<double,
 * Dynamic, Dynamic>), cells n x ncols with the column order of
 * ABM-3d/ABM-3d-cpp/include/indices.hpp:17-47 (+ gamma in column 21 when
 * cell-cell adhesion is on), neighbor rows m x 7 (i, j, dx, dy, dz, si, sj).
 *
 * Ownership: the caller owns every host buffer; a context owns its device
 * buffers, its CUDA stream and its CUDA graphs.  A context is not thread-safe;
 * use one context per host thread.  Every call returns ABM_OK (0) or a negative
 * status; abm_last_error() gives the message.  No call falls back to the CPU:
 * without a usable CUDA device abm_create() fails with ABM_ERR_CUDA.
 */
#ifndef ABM_CAPI_H
#define ABM_CAPI_H

#ifdef __cplusplus
extern "C" {
#endif

#define ABM_OK 0
#define ABM_ERR_ARG -1          /* invalid argument or unsupported option */
#define ABM_ERR_CUDA -2         /* CUDA runtime error (device missing, launch failure, ...) */
#define ABM_ERR_CAPACITY -3     /* a device capacity (cells, neighbors per cell, bins) was exceeded */
#define ABM_ERR_NAN -4          /* NaN/Inf in forces, velocities or the error norm */
#define ABM_ERR_STATE -5        /* call order violated (e.g. iterate before upload) */

/* Integration modes, as IntegrationMode in simulation.hpp:45-55 */
#define ABM_VELOCITY_VERLET 0   /* 3-D, FP64, reference controller; needs abm_params.M0 > 0 */
#define ABM_HEUN_EULER 1
#define ABM_BOGACKI_SHAMPINE 2
#define ABM_RUNGE_KUTTA_FEHLBERG 3
#define ABM_DORMAND_PRINCE 4

/* Step-size controllers.  REFERENCE: the rule of simulation.hpp:1688-1769 (trial, up to
 * max_tries retries, a final re-run accepted unconditionally).  PI and LEARNED propose
 * the dt of every iteration's first attempt, which is accepted as is when its embedded
 * error passes (E <= 1); otherwise the REFERENCE rule continues from that attempt (its
 * retries and final re-run).  PI: after each accepted step of dt with scaled error E_n,
 * the next dt is dt 0.9 E_n^(-0.7/k) E_(n-1)^(0.4/k), k = error order + 1 (E_(n-1) = 1
 * before the second step), the factor held to [0.2, 10] and dt to [min_stepsize,
 * max_stepsize].  LEARNED: the step-size network adds its output to that same PI ratio
 * (below), so a network whose output is zero is the PI controller, and after a failed
 * first attempt among the last 8 steps the network may only shorten the PI step. */
#define ABM_CONTROLLER_REFERENCE 0
#define ABM_CONTROLLER_LEARNED 1
#define ABM_CONTROLLER_PI 2

/* Step-size network: 32 features -> 64 -> 64 -> 1 (ReLU), output ln(dt / dt_prev).
 * Flat FP32 parameter layout: W1[64][32], b1[64], W2[64][64], b2[64], w3[64], b3. */
#define ABM_MLP_FEATURES 32
#define ABM_MLP_HIDDEN 64
#define ABM_MLP_NPARAM 6337
/* The proposal is ln(dt / dt_prev) = clamp(b + y, ln 0.2, ln 10): y the network output,
 * b = ln 0.9 - (0.7 ln E_last - 0.4 ln E_prev)/(q+1) the PI ratio (E_last, E_prev: scaled
 * errors of the last two accepted steps, q: error order of the tableau).
 * Log row: 32 features, ln(dt_max / dt_first) with dt_max = dt_first E^(-1/(q+1)),
 * ln(dt_first / dt_prev), log10 E of the first attempt, 1 if it passed (E <= 1), b, and
 * three spare columns. */
#define ABM_MLP_LOG_COLS 40

#define ABM_PRECISION_FP64 0    /* everything in FP64 */
#define ABM_PRECISION_MIXED 1   /* segment distance + pair force in FP32; near-parallel branch,
                                   positions, orientations, stage sums and error norm in FP64 */

typedef struct abm_params {
    /* geometry and mechanics (runSimulation arguments, simulation.hpp:1106-1165) */
    double R, Rcell, E0, Ecell;
    double L0, Ldiv;
    double neighbor_threshold;   /* abmConstAdhesion.cpp:53: 0.5 (2R + Ldiv) */
    double nz_threshold;
    int adhesion_mode;           /* 0 = NONE, 1 = JKR_ISOTROPIC with a fixed-gamma radius table */
    int integration_mode;        /* ABM_VELOCITY_VERLET, ABM_HEUN_EULER ... ABM_DORMAND_PRINCE */
    double max_stepsize, min_stepsize;
    double max_error_allowed, min_error;
    int max_tries_update_stepsize;
    int iter_update_stepsize, iter_update_neighbors;
    double max_rxy_noise, max_rz_noise, max_nxy_noise, max_nz_noise;
    double cell_surface_coulomb_coeff;
    int no_surface;
    /* growth and division (growth.hpp:51-426) */
    double growth_mean, growth_std, daughter_length_std;
    double daughter_angle_xy_bound, daughter_angle_z_bound;
    unsigned long long rng_seed;
    /* device-side choices */
    int precision;               /* ABM_PRECISION_FP64 or ABM_PRECISION_MIXED */
    int cap_cells;               /* device capacity in cells (>= the largest population) */
    int cap_neighbors_per_cell;  /* directed neighbor slots per cell (0 = default: 192 in 3-D, 64 in 2-D) */
    int pair_lanes;              /* lanes per cell of the no-alloc entry point's pair kernel: 4, 8, 16 or 32 (0 = 8) */
    int use_graphs;              /* 1 = capture the iteration in a CUDA graph */
    /* step-size control (no reference counterpart beyond ABM_CONTROLLER_REFERENCE) */
    int controller;              /* ABM_CONTROLLER_REFERENCE, ABM_CONTROLLER_LEARNED or ABM_CONTROLLER_PI */
    int stepsize_log_capacity;   /* rows of step-size features logged per context (0 = off) */
    /* model dimension: 3 (ABM-3d, default when 0) or 2 (ABM-2d).  The 2-D model uses the
     * 17-column cell layout of ABM-2d/ABM-2d-cpp/include/indices.hpp, neighbor rows
     * (i, j, dx, dy, si, sj), n x 4 forces / velocities / errors, Hertz prefactors of
     * 2D/include/simulation.hpp:232-235, adhesion_mode 1 = JKR-Lagrange
     * (2D/include/adhesion.hpp:403-448, strength and mindist below), composite drag with
     * rho_c = (sigma0 R^2 / 4 E0)^(1/3), uniform noise max_noise on (r, n), and
     * daughter_angle_xy_bound as its daughter angle bound (daughter_angle_z_bound must be 0).
     * integration_mode ABM_BOGACKI_SHAMPINE (the 2-D driver's) or ABM_HEUN_EULER. */
    int dims;
    double sigma0;
    double adhesion_strength, adhesion_mindist;
    double max_noise;
    /* shape of the screened pair pass: the least pairs per block (512..2048, 0 = 1024)
     * and the most blocks per SM (0 = as many as are resident at once);
     * abm_autotune_pair_tile picks them */
    int pair_tile, pair_blocks_per_sm;
    /* skin of the active pair list in um (0 = 0.3, negative = none): pairs farther than
     * 2R + skin at a refresh are skipped until the cells may have moved by half the skin */
    double pair_skin;
    /* where each cell's pair shares are summed: 1 = inside the first RK attempt,
     * 2 = a separate light kernel before it (0 = 1, the faster on B200) */
    int pair_sum;
    /* cell-cell kinetic friction (3-D, FP64): 0 = NONE, 1 = KINETIC (mechanics.hpp:61-65,
     * 1031-1175), the coefficient of each cell in column 22 with adhesion, 21 without
     * (simulation.hpp:1184-1186); its norm capped at cell_cell_coulomb_coeff (4/3) E0
     * sqrt(R/2) overlap^(3/2) when that coefficient is positive (runSimulation's default 1) */
    int friction_mode;
    double cell_cell_coulomb_coeff;
    /* integration_mode ABM_VELOCITY_VERLET (0): the cell mass at length L0, which sets the
     * density of every cell (simulation.hpp:1279-1290); must be positive in that mode */
    double M0;
} abm_params;

typedef struct abm_stats {
    long long iterations;        /* accepted steps taken by abm_iterate */
    long long attempts;          /* RK evaluations (stepRungeKuttaAdaptive calls) */
    long long retries;           /* controller re-runs at a reduced step (simulation.hpp:1717) */
    long long rebuilds;          /* neighbor-table rebuilds */
    long long divisions;         /* cells divided */
    double t, dt;                /* simulated time and current step size */
    double last_max_error;       /* scaled max error of the accepted attempt */
    int n_cells, n_pairs;        /* current population and neighbor pairs (unordered) */
    long long rejected;          /* iterations whose first attempt failed the error test */
    long long log_rows;          /* step-size feature rows written so far */
    long long cell_steps;        /* sum of the population over accepted steps */
} abm_stats;

/* Device time per kernel group, from CUDA events on the context stream. */
typedef struct abm_profile {
    double pair_force_ms;        /* cellCellInteractionForces (+ distance refresh) */
    double attempt_ms;           /* all RK attempts incl. controller and growth */
    double rebuild_ms;           /* getCellNeighbors rebuilds */
    long long pair_force_launches, attempt_launches, rebuild_launches;
    long long iterations;
} abm_profile;

typedef struct abm_ctx abm_ctx;

/* Create a context on the current CUDA device.  No reference counterpart: the
 * reference keeps this state on the stack of runSimulation (simulation.hpp:1106-1170).
 * On a failure other than ABM_ERR_ARG for a NULL argument, *ctx still receives a
 * context that holds the reason (abm_last_error); release it with abm_destroy. */
int abm_create(const abm_params* params, abm_ctx** ctx);
int abm_destroy(abm_ctx* ctx);
const char* abm_last_error(const abm_ctx* ctx);
/* The context's CUDA stream (cudaStream_t), for callers that order their own work after it. */
int abm_get_stream(abm_ctx* ctx, void** stream);
int abm_synchronize(abm_ctx* ctx);

/* JKR contact radius, the larger root of the jkr.hpp:67-144 quartic (jkrContactRadius(...).second). */
int abm_jkr_contact_radius(double delta, double Req, double E, double gamma, double* radius);
/* Radius table over LinSpaced(n, 0, 2 (R - Rcell)): calculateJKRContactRadii, simulation.hpp:86-104
 * with the mesh of simulation.hpp:1379-1382. */
int abm_jkr_radius_table(double R, double Rcell, double E0, double gamma, int n_mesh,
                         double* delta_out, double* radius_out);
/* jkrOptimalSurfaceEnergyDensity (jkr.hpp:1369-1407) as runSimulation calls it
 * (simulation.hpp:1354-1358): the adhesion energy density whose JKR force balance puts two
 * cells at centerline distance eqdist, in closed form.  ABM_ERR_ARG unless
 * 2 Rcell <= eqdist < 2 R (the reference caps the overlap at 2 (R - Rcell)). */
int abm_jkr_optimal_gamma(double R, double Rcell, double E0, double eqdist, double* gamma);
/* Install the fixed-gamma table (IsotropicJKRDataFixedGamma, mechanics.hpp:113-153). */
int abm_set_jkr_table(abm_ctx* ctx, const double* delta, const double* radius, int n);
/* Radius table over LinSpaced(n_delta, 0, 2 (R - Rcell)) x LinSpaced(n_gamma, 0, max_gamma),
 * overlap-major (radius_out[i * n_gamma + j] at delta_out[i], gamma_out[j]):
 * calculateJKRContactRadii over two meshes, simulation.hpp:120-145. */
int abm_jkr_radius_table_variable(double R, double Rcell, double E0, double max_gamma, int n_delta, int n_gamma,
                                  double* delta_out, double* gamma_out, double* radius_out);
/* Install a variable-gamma table (IsotropicJKRDataVariableGamma, mechanics.hpp:159-199): the
 * cell-cell JKR force of a pair with gamma = min(gamma_i, gamma_j) > 0 then takes its contact
 * radius by bilinear interpolation on the (overlap, gamma) mesh (forcesIsotropicJKRLagrange,
 * adhesion.hpp:412-526); a gamma beyond the mesh takes the end cell.  radius is overlap-major,
 * n_delta x n_gamma; both meshes strictly increasing.  abm_set_jkr_table removes it. */
int abm_set_jkr_table_variable(abm_ctx* ctx, const double* delta, int n_delta, const double* gamma, int n_gamma,
                               const double* radius);

/* Phenotype switching between groups 1 and 2 (3-D), applied inside abm_iterate after each
 * accepted step, after basal-only compaction and the periodic neighbor rebuild
 * (simulation.hpp:1866-2022).  Replaces the switching arguments of runSimulation
 * (simulation.hpp:1135-1160: switch_mode, switch_rates, growth_means / growth_stds,
 * switch_attributes, attribute_values, switch_timescale, max_gamma, modulate_local_viscosity,
 * viscosity_lims, max_coordination_number).
 *   mode        0 none, 1 Markov (switch.hpp:45-95), 2 inherited at division (switch.hpp:97-142)
 *   n_start     switching starts once the colony has this many cells
 *   rates       2 x 2 row-major, row = current group: rates per unit time (Markov) or
 *               probabilities (inherited)
 *   growth_mean, growth_std   growth-rate distribution of each group; with switching on,
 *               daughters draw from their mother's group's (growth.hpp:634-644)
 *   timescale   ramp time of the switched attributes and gamma; 0 = at once
 *   n_attr, attr_col, attr_targets   up to 4 switched attributes, columns 17 (eta0),
 *               18 (eta1) or 19 (sigma0), with targets 2 x n_attr row-major (group 1, group 2)
 *   max_gamma   gamma ramps to max_gamma in group 1, to 0 in group 2 (adhesion on)
 *   modulate, visc_lims, max_coord   local viscosity (adhesion on): eta0 between
 *               visc_lims (min, max of group 1, then of group 2) by the share of group-1 cells
 *               among the contacts, saturating at max_coord of them (simulation.hpp:1958-2020)
 * Random draws: the Philox policy of the division and noise kernels, purpose SWITCH, counters
 * (iteration, cell or division pair, slot).  ABM_ERR_STATE for a 2-D context. */
int abm_set_switching(abm_ctx* ctx, int mode, int n_start, const double* rates, const double* growth_mean,
                      const double* growth_std, double timescale, int n_attr, const int* attr_col,
                      const double* attr_targets, double max_gamma, int modulate, const double* visc_lims,
                      int max_coord);
/* Basal-only growth (simulation.hpp:1831-1856): with the surface present, after each accepted
 * step only the cells whose deepest overlap R - rz + half_l nz exceeds min_overlap stay (in
 * order), followed by a neighbor rebuild when any was dropped. */
int abm_set_basal_only(abm_ctx* ctx, int basal_only, double min_overlap);
/* Cells dropped by basal-only compaction since the context was created. */
int abm_basal_dropped(abm_ctx* ctx, long long* dropped);

/* Cell state in and out (the cells array of runSimulation).  ld >= n. */
int abm_upload_cells(abm_ctx* ctx, const double* colmajor, int n, int ncols, int ld);
int abm_download_cells(abm_ctx* ctx, double* colmajor, int ld);
int abm_get_num_cells(abm_ctx* ctx, int* n);
/* Simulation clock (t, dt, iter of runSimulation, simulation.hpp:1166-1168). */
int abm_set_clock(abm_ctx* ctx, double t, double dt, int iter);
int abm_get_clock(abm_ctx* ctx, double* t, double* dt, int* iter);
/* Lineage vector (parents) of runSimulation; cell IDs index it. */
int abm_set_parents(abm_ctx* ctx, const int* parents, int n);
int abm_get_parents(abm_ctx* ctx, int* out, int cap, int* n);

/* getCellNeighbors (mechanics.hpp:520-593): rebuild the neighbor pair set with a
 * uniform-grid cell list; *m receives the number of unordered pairs. */
int abm_build_neighbors(abm_ctx* ctx, int* m);
/* The table in the reference's row order (i ascending, then j < i ascending),
 * m x 7 column-major with leading dimension ld >= m.  Distances are those of
 * updateNeighborDistances (mechanics.hpp:604-648) on the current cells. */
int abm_download_neighbors(abm_ctx* ctx, double* rows, int ld, int cap, int* m);
/* Replace the pair set by the given rows (columns 0 and 1 are read). */
int abm_upload_neighbors(abm_ctx* ctx, const double* rows, int m, int ld);

/* cellCellInteractionForces (mechanics.hpp:1209-1350, 1390-1659): dE/dq, n x 6. */
int abm_cell_cell_forces(abm_ctx* ctx, double* dEdq_colmajor);
/* getVelocities (mechanics.hpp:2011-2347) of the current cells, no noise: n x 6. */
int abm_get_velocities(abm_ctx* ctx, double* v_colmajor);
/* stepRungeKuttaAdaptive (mechanics.hpp:2406-2612) at dt without accepting it.
 * Optional outputs: the new cell array (n x ncols), the error array (n x 6) and
 * the controller's scaled max error (simulation.hpp:1697-1705).  `attempt`
 * selects the noise stream. */
int abm_rk_attempt(abm_ctx* ctx, double dt, int attempt, double* cells_out,
                   double* errors_out, double* max_scaled_error);
/* growCells (growth.hpp:51-57). */
int abm_grow(abm_ctx* ctx, double dt);
/* divideMaxLength + divideCells (growth.hpp:66-71, 166-426) at the current clock;
 * *n_divided receives the number of mothers. */
int abm_divide(abm_ctx* ctx, int* n_divided);
/* Number of tries the last division took (the ntries loop of growth.hpp:252-398). */
int abm_last_division_tries(abm_ctx* ctx, int* tries);

/* n_iters iterations of the runSimulation loop body (simulation.hpp:1617-1864):
 * divide -> rebuild if divided -> adaptive RK step with the step-size
 * controller -> grow -> refresh distances -> t, iter -> rebuild every
 * iter_update_neighbors.  Stops early when n_cells_stop > 0 and the population
 * reaches it.  Runs asynchronously on the context stream; stats (optional)
 * forces a synchronisation. */
int abm_iterate(abm_ctx* ctx, int n_iters, int n_cells_stop, abm_stats* stats);
int abm_get_stats(abm_ctx* ctx, abm_stats* stats);
/* "conditional" when the iteration graph uses IF/WHILE nodes, otherwise why it could not
 * (the fallback graph launches every retry and decides division on the host). */
const char* abm_graph_info(const abm_ctx* ctx);
/* Same as abm_iterate without graphs, with CUDA events around each kernel group
 * (no reference counterpart; measurement only). */
int abm_profile_iterations(abm_ctx* ctx, int n_iters, abm_profile* profile);

/* 2-D adhesion flags (the to_adhere array of 2D/include/simulation.hpp:242-258), one per
 * neighbor row in the order of abm_download_neighbors.  abm_build_neighbors and every
 * rebuild set them from the distances at that time, as the reference does. */
int abm_get_adhesion_flags(abm_ctx* ctx, int* flags, int cap, int* m);
int abm_set_adhesion_flags(abm_ctx* ctx, const int* flags, int m);

/* Stop on the device once the population reaches n_max cells (0 = no limit): the
 * terminate() test at the top of the loop (simulation.hpp:1600-1615); a context at its
 * limit takes no further division or step.  Used by batches, where the host does not
 * poll each context. */
int abm_set_cell_limit(abm_ctx* ctx, int n_max);

/* ---------------------------------------------------------------------------
 * Batches (no reference counterpart: the reference runs replicates as separate jobs).
 * A batch advances independent contexts (replicate biofilms of any sizes, each with
 * its own clock, step size and controller) by one CUDA graph launch per iteration:
 * every context's iteration graph is a branch of one graph, so a context's results
 * are bit-identical to advancing it alone.  Contexts must share a device and
 * iter_update_neighbors.  Batch calls report errors through abm_batch_last_error().
 * ------------------------------------------------------------------------- */
typedef struct abm_batch abm_batch;
int abm_batch_create(abm_ctx* const* ctxs, int n, abm_batch** batch);
int abm_batch_iterate(abm_batch* batch, int n_iters);
int abm_batch_synchronize(abm_batch* batch);
int abm_batch_get_stream(abm_batch* batch, void** stream);
int abm_batch_destroy(abm_batch* batch);
const char* abm_batch_last_error(void);
/* Autotuner of the screened pair pass: times tiles of at least 512, 1024 and 2048 pairs per
 * block with at most 1, 2 and 4 blocks per SM (9 candidates, c = 3 * tile index + grid
 * index) on a scratch context holding `cells`, over `launches` launches each, and
 * returns the fastest shape; ms_per_launch (9 entries, may be NULL) receives each time. */
int abm_autotune_pair_tile(const abm_params* params, const double* cells, int n, int ncols, int ld,
                           const double* jkr_delta, const double* jkr_radius, int jkr_n, int launches,
                           int* best_tile, int* best_blocks_per_sm, float* ms_per_launch);

/* ---------------------------------------------------------------------------
 * Step-size network (no reference counterpart).  The weights are the flat FP32
 * layout above; every kernel rounds them to BF16 and accumulates in FP32 on the
 * tensor cores.
 * ------------------------------------------------------------------------- */
/* Install / read the weights the context's learned controller uses. */
int abm_stepsize_set_weights(abm_ctx* ctx, const float* weights, int n_param);
int abm_stepsize_get_weights(abm_ctx* ctx, float* weights, int n_param);
/* Copy the logged rows (ABM_MLP_LOG_COLS floats each, oldest first, at most
 * stepsize_log_capacity) into rows[cap_rows][ABM_MLP_LOG_COLS]; n_rows = rows copied. */
int abm_stepsize_get_log(abm_ctx* ctx, float* rows, int cap_rows, int* n_rows);
int abm_stepsize_clear_log(abm_ctx* ctx);
/* Host-buffer entry points on the current device (they allocate device memory).
 * X is n x 32 row-major; Y and T have n entries. */
int abm_mlp_forward(const float* weights, const float* X, int n, float* Y);
/* Gradient of L = 0.5/n sum (y - t)^2 with respect to the weights, and L. */
int abm_mlp_grad(const float* weights, const float* X, const float* T, int n, float* grad, float* loss);
/* Mini-batch Adam (batches of 64, seeded order) on the GPU; weights in/out;
 * loss_per_epoch (epochs entries, may be NULL) gets each epoch's mean loss. */
int abm_mlp_train(float* weights, const float* X, const float* T, int n, int epochs, float lr,
                  unsigned seed, float* loss_per_epoch);
const char* abm_mlp_last_error(void);

/* ---------------------------------------------------------------------------
 * Cell-cell forces without device allocation.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: their device memory is owned by
 * another allocator (a framework's caching pool or a fixed budget), or they
 * cannot take the device-wide synchronisation of cudaMalloc/cudaFree inside a
 * step loop.  Same result as abm_cell_cell_forces (dE/dq, mechanics.hpp:
 * 1209-1659) for a neighbor set given in CSR form: d_row_ptr[n + 1] and
 * d_col[n_entries] list each cell's neighbors in both directions, each row
 * sorted ascending.  d_cells (n x ncols, leading dimension ld), the CSR arrays
 * and d_dEdq (n x 6, leading dimension n) are device buffers the caller owns;
 * jkr_delta / jkr_radius are host arrays (ignored without adhesion), read during
 * the call only: they travel to the device inside the launch parameters.  Work is
 * enqueued on `stream` (a cudaStream_t, 0 = legacy default stream); results are
 * ready when the stream reaches that point.  3-D model only (dims 0 or 3);
 * adhesion_mode 0 or 1; precision ABM_PRECISION_FP64 or ABM_PRECISION_MIXED.
 *
 * Scratch lives in one fixed __device__ array of about 21 MB that every GPU
 * loading this library holds until the process exits.  Limits per call:
 * n <= ABM_NOALLOC_MAX_CELLS, n_entries <= ABM_NOALLOC_MAX_ENTRIES; larger
 * inputs return ABM_ERR_CAPACITY.  The first call on a device looks up the
 * array's address (cudaGetSymbolAddress) with that device current: make it
 * before any stream capture.  All calls share the array, so calls that overlap
 * on the GPU race; serialise them.  The call allocates nothing.
 * abm_noalloc_last_error() describes the last failure of this thread.
 *
 * The CSR is checked on the device before any kernel indexes with it: row_ptr[0]
 * = 0, row_ptr[n] = n_entries, rows non-decreasing, columns in [0, n) and not the
 * row itself, rows strictly ascending, and every entry (i, j) matched by (j, i).
 * A CSR that fails is never used to index memory: the call fills d_dEdq with NaN,
 * and abm_cell_cell_forces_noalloc_status then returns ABM_ERR_ARG with the
 * reason in abm_noalloc_last_error().
 * ------------------------------------------------------------------------- */
#define ABM_NOALLOC_MAX_CELLS 32768
#define ABM_NOALLOC_MAX_ENTRIES 524288
int abm_cell_cell_forces_noalloc(const abm_params* params, const double* d_cells, int n, int ncols, int ld,
                                 const int* d_row_ptr, const int* d_col, int n_entries,
                                 const double* jkr_delta, const double* jkr_radius, int jkr_n,
                                 double* d_dEdq, void* stream);
/* Waits for `stream` and reports whether the CSR of the last abm_cell_cell_forces_noalloc
 * call on the current device passed its device-side check: ABM_OK, or ABM_ERR_ARG. */
int abm_cell_cell_forces_noalloc_status(void* stream);
const char* abm_noalloc_last_error(void);

/* ---------------------------------------------------------------------------
 * Frame and lineage files in the reference's text formats, so that a run driven
 * through abm_iterate writes what runSimulation writes.  Host code, no device
 * memory.  Arrays are column-major; abm_io_last_error() describes the last failure
 * of this thread.
 * ------------------------------------------------------------------------- */
/* writeCells (utils.hpp:153-198 of both models): `params` holds "key = value" lines
 * (each written as "# key = value"; NULL for none); the ID and group columns (3-D 0
 * and 20, 2-D 0 and 16 by `dims`) are written as integers and the columns between
 * them as doubles with 10 significant digits; further columns only if listed in
 * extra_cols, as integers (extra_types 0) or doubles (1), like write_other_cols. */
int abm_write_cells(const char* path, const double* cells, int n, int ncols, int ld, int dims,
                    const char* params, const int* extra_cols, const int* extra_types, int n_extra);
/* readCells (utils.hpp:96-139): rows into `cells` (column-major, leading dimension
 * cap_rows), parameters into `params` as "key = value" lines (may be NULL).  With
 * cells == NULL only *n and *ncols are set (the sizes to allocate). */
int abm_read_cells(const char* path, double* cells, int cap_rows, int cap_cols, int* n, int* ncols,
                   char* params, int params_cap);
/* writeLineage (utils.hpp:296-311): "i<TAB>parents[i]" for i < n. */
int abm_write_lineage(const char* path, const int* parents, int n);
/* readLineage (utils.hpp:265-287): parents[child] = parent; *n = largest child ID + 1.
 * Entries for IDs the file does not list are left as the caller set them (the reference
 * returns a map).  With parents == NULL only *n is set. */
int abm_read_lineage(const char* path, int* parents, int cap, int* n);
const char* abm_io_last_error(void);

/* Frames of a device-resident run (runSimulation's dt_write writes,
 * simulation.hpp:2025-2058): with dt_write > 0 and slots > 0, an accepted step
 * whose time crosses a multiple of dt_write marks a frame, and the end of that
 * iteration copies the cells into a ring of `slots` snapshots on the device, so the
 * loop keeps running without host round trips.  Turning frames on or off, or
 * changing the slot count, rebuilds the iteration graph; the frame count restarts at
 * 0.  dt_write = 0 or slots = 0 turns them off.  A context in a batch takes its
 * frame setting into the batch's graph at abm_batch_create: set frames before
 * creating the batch and leave them unchanged while the batch exists. */
int abm_set_frames(abm_ctx* ctx, double dt_write, int slots);
/* frames marked since abm_set_frames (the ring keeps the last `slots` of them) */
int abm_frames_taken(abm_ctx* ctx, int* taken);
/* frame `index` (0-based): its cells (column-major, cells-array layout; NULL for the
 * sizes only), cell count, time, iteration and lineage length at that step.
 * ABM_ERR_CAPACITY when the ring has overwritten it. */
int abm_download_frame(abm_ctx* ctx, int index, double* cells, int ld, int* n, double* t, int* iter,
                       int* n_parents);

/* Exact binary checkpoints: the resume the reference makes from its text frames
 * (readCells and readLineage, utils.hpp:96-139 and 265-287, whose 10-digit values
 * move a resumed run off its course), without the rounding.  A checkpoint holds the
 * FP64 cells, the neighbor set, the lineage, the clock and what the step-size
 * controllers carry between iterations (the last steps' dt, scaled errors and
 * accept flags, the network's step statistics, the loop's counters).  Save at an
 * iteration boundary (between abm_iterate calls) after the neighbors exist; load
 * into a context created with the same parameters, JKR table and network weights,
 * and it continues bit for bit as the saved run would.  Frames, the cell limit and
 * switching settings are not part of it: set them again.  Host byte order;
 * ABM_ERR_ARG for a file that is not a complete checkpoint of this library or
 * belongs to the other model, ABM_ERR_CAPACITY when it holds more than cap_cells. */
int abm_save_checkpoint(abm_ctx* ctx, const char* path);
int abm_load_checkpoint(abm_ctx* ctx, const char* path);

#ifdef __cplusplus
}
#endif
#endif /* ABM_CAPI_H */
