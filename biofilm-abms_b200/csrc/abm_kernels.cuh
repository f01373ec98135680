// Kernel-side shared types and launch wrappers of the B200 mechanics step.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "abm_device.cuh"

namespace abm {

const int MAX_STAGES = 7;

// Controller modes of one iteration (simulation.hpp:1690-1769)
// MODE_COMMIT: the learned controller's proposal passed the error test; the final
// attempt copies its candidate state instead of re-running the step.
enum CtrlMode { MODE_TRIAL = 0, MODE_RETRY = 1, MODE_FINAL = 2, MODE_COMMIT = 3 };

// Step-size network: 32 features -> 64 -> 64 -> 1 (log dt ratio)
const int MLP_IN = 32, MLP_H = 64;
const int MLP_OFF_W1 = 0, MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_IN, MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
const int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H, MLP_OFF_W3 = MLP_OFF_B2 + MLP_H, MLP_OFF_B3 = MLP_OFF_W3 + MLP_H;
const int MLP_NPARAM = MLP_OFF_B3 + 1;
// log row: 32 features, ln(dt_max / dt_first), ln(dt_first / dt_prev), log10 E, passed,
// the proposal's error-model baseline, 3 spare columns
const int MLP_LOG_COLS = 40;
const int HIST = 8;
const int STAT_V2_SHIFT = 20, STAT_G_SHIFT = 32;

// Status bits raised on the device and turned into ABM_ERR_* by the host.
enum StatusBits {
    ST_NAN = 1,            // NaN/Inf in the error norm or velocities
    ST_NBR_OVERFLOW = 2,   // more neighbors than cap_neighbors_per_cell
    ST_BIN_OVERFLOW = 4,   // grid needs more bins than allocated
    ST_CELL_OVERFLOW = 8,  // division would exceed cap_cells
};

// Device-resident clock, controller and population state.
struct Ctrl {
    double t, dt;               // simulated time, current step size
    double dt_try;              // step size of the next attempt
    double factor;              // controller factor (simulation.hpp:1710-1757)
    double last_max_error;
    double last_trial_error;
    unsigned long long err_bits;    // max scaled error of the running attempt (ordered bits)
    unsigned int blocks_done;       // last-block counter of the running attempt
    int iter;
    int mode;                   // CtrlMode
    int tries;                  // j in simulation.hpp:1716
    int attempt;                // attempt index within the iteration (noise stream)
    int status;                 // StatusBits
    int n;                      // cells
    int n_dir;                  // directed neighbor entries (2 x pairs)
    int n_divide;               // mothers in the pending division
    long long attempts, retries, iterations, rebuilds, divisions;
    unsigned long long eval_err_bits;   // scaled max error of the last API attempt
    // division bookkeeping (growth.hpp:166-426)
    int div_count;              // running count of flagged / satisfied cells
    unsigned int div_blocks;    // last-block counter of the division kernels
    int div_done, div_tries, last_div_tries;
    int n_parents;              // length of the lineage vector
    long long div_events;       // iterations in which cells divided
    // step-size features (filled when StepParams::stats_on)
    // sums in fixed point so that their value does not depend on the order of the atomics
    unsigned long long st_vmax_bits;    // max |v_r| of the last accepted step (ordered bits)
    unsigned long long st_ovl_bits[2];  // max overlap of the pair-force passes of even / odd iterations
    unsigned long long st_v2_fx;        // sum |v_r|^2 * 2^STAT_V2_SHIFT
    unsigned long long st_g_fx;         // sum of growth rates * 2^STAT_G_SHIFT
    unsigned long long st_near_div;     // cells with l > 0.9 Ldiv
    int since_div;                      // iterations since cells last divided
    double hist_dt[HIST], hist_err[HIST];   // accepted dt and its scaled error, newest at hist_pos - 1
    int hist_acc[HIST];                 // 1 if that iteration's first attempt passed the error test
    int hist_pos;
    int first_passed;                   // the running iteration's first attempt passed
    double dt_prev;                     // accepted dt before the running iteration
    long long rejected;                 // iterations whose first attempt failed the error test
    long long log_rows;                 // feature rows written (ring position = log_rows % capacity)
    // cell-count stop on the device (terminate(), simulation.hpp:1600-1615): decided at the
    // start of each iteration by the division count; a halted context skips its iterations
    int halt_n;                         // 0 = no limit
    int halted;
    long long cell_steps;               // sum of the population over accepted steps
    // screened pair pass: the active list (pairs that passed the bound test with the
    // skin at the last refresh) and the motion since then
    int n_surv;                         // active pairs
    int n_surv_next;                    // pairs appended by a refresh in progress
    int screen_valid;                   // 0 after a rebuild, an upload or a division
    unsigned int surv_blocks;           // last-block counter of the pair pass
    int n_order;                        // cells covered by the attempt order (0: index order)
    // frames: an accepted step whose time crosses a multiple of dt_write marks a frame,
    // which the snapshot kernel at the end of the iteration copies into a ring slot
    double dt_write;                    // 0: no frames
    int frame_due, frames_taken;
    unsigned int frame_blocks;          // last-block counter of the snapshot kernel
    // friction: candidate pairs of the last pair pass, pairs whose decisions change with the
    // stage, and the trial loop's state (a trial pass is pending; a check changed a decision)
    int fr_ncand, fr_ncand_next;
    int fr_nflip, fr_nflip_next;
    int fr_pending, fr_changed;
    unsigned int fr_blocks;
    // basal-only compaction: cells kept by the last test, cells dropped so far
    int n_keep;
    long long basal_dropped;
    double drift;                       // sum over accepted steps of the max segment motion
    unsigned long long drift_bits;      // block maxima of the running attempt (ordered bits)
};

struct Grid {
    double x0, y0, z0, edge, inv_edge;
    int nx, ny, nz, nbins;
    double max_half_l;
};

struct StepParams {
    MechParams mp;
    int s;                      // stages
    double A[MAX_STAGES][MAX_STAGES], b[MAX_STAGES], bs[MAX_STAGES];
    double inv_q1;              // 1 / (error_order + 1)
    double tol, min_error, min_stepsize, max_stepsize;
    int max_tries, iter_update_stepsize;
    double noise_max[6];
    int noise_on;
    uint64_t seed;
    // 2-D model: composite drag eta0 + eta1 rho_c / R (2D/include/mechanics.hpp:264-279)
    double rho_c;
    double max_noise_2d;
    // step-size control
    int propose;                // 1: every iteration's first attempt runs at a proposed dt and is
                                // accepted as is when its error passes (learned and PI controllers)
    int network;                // 1: the step-size network makes the proposal (learned controller)
    int pi;                     // 1: the PI rule makes the proposal after each accepted step
    int mixed;                  // 1: mixed precision (3-D): cells in surface contact take the FP32
                                // contact branch of the velocity solve
    int fric;                   // 1: cell-cell kinetic friction (3-D, FP64)
    int stats_on;               // accumulate the network's features (learned or logging)
    double near_div_length;     // 0.9 Ldiv
    double4* stat_part;         // per-block (max |v_r|, sum |v_r|^2, sum growth, near-division count)
    float* log_buf;             // MLP_LOG_COLS floats per row, log_cap rows (ring)
    int log_cap;
    const int* order;           // attempt order of the first ctrl->n_order cells (3-D), or null
};

struct ForceParams {
    double R, Rcell, E0;
    double pf0, pf1, pf2;       // repulsion prefactors (simulation.hpp:1270-1274)
    double max_overlap;         // 2 (R - Rcell)
    int adhesion;
    int jkr_n;
    double jkr_step;            // spacing of the overlap mesh
    // variable-gamma table (IsotropicJKRDataVariableGamma, mechanics.hpp:159-199): radii on
    // the overlap mesh x the gamma mesh, overlap-major; jkr_ng = 0 without it
    int jkr_ng;
    double jkr_gstep;           // spacing of the gamma mesh
    const double* jkr_gam;      // gamma mesh (jkr_ng)
    const double* jkr_rad2;     // radii (jkr_n x jkr_ng)
    int stats;                  // record the max overlap (step-size features)
    double skin;                // screened pair pass: margin of the active list (um)
    // 2-D model (ABM-2d): Hertz prefactors of 2D/include/simulation.hpp:232-235 and
    // the JKR-Lagrange adhesion of 2D/include/adhesion.hpp:403-448
    double pf2d[3];
    double adh_strength, adh_mindist;
    const unsigned char* adhere;    // per CSR entry: to_adhere at the last rebuild
    // cell-cell kinetic friction (cellCellFrictionForces, mechanics.hpp:1031-1175), FP64, 3-D
    int fric;
    int surface;                    // a surface is present (the planar-contact rule applies)
    double coulomb_cc;              // Coulomb cap coefficient (not positive: no cap)
    const Vel* vel;                 // stored velocities of the cells (dr, dn)
    const double* feta;             // friction coefficient of each cell
    double4* fbuf;                  // per CSR entry: share change when the contact is planar
    int* fmask;                     // per CSR entry: FR_* bits
    int* fr_list;                   // pairs with a planar-contact candidate, this pass
};

// Friction: a contact with |dz / d| < 1e-3 whose two contact points lie below 1.01 R is taken
// in the xy-plane (mechanics.hpp:1090-1110).  The positions enter only through that test, so
// an attempt's pair forces are fixed but for those candidate pairs, whose planar decision can
// change from stage to stage.  Per CSR entry: FR_CAND, FR_D0 = the decision at y0, and bits
// 0-7 = the stages whose decision differs from FR_D0.
const int FR_CAND = 1 << 16, FR_D0 = 1 << 17, FR_FLIPS = 0xFF;

struct BuildParams {
    double threshold;           // neighbor_threshold
    double prefilter;           // neighbor_threshold + Ldiv + 2 R (mechanics.hpp:551)
    int cap_per_cell;
};

// Where an attempt finds the pair force when it completes the sum itself:
// fused = 1: fcc holds the lower-neighbor share, jbuf the partners' shares;
// fused = 2: jbuf holds both shares of every pair (screened pass), as double4;
// fused = 3: the same as float4 (mixed precision);
// fused = 0: fcc already holds the total.
struct PairGather {
    int fused;
    const int* row_ptr;
    const int* lower_end;
    const double4* jbuf;
    Gen6* fcc_w;
    // friction: the planar-contact corrections of each stage, and the stage states of the
    // cells with candidate contacts (z and n_z per stage, written by the trial passes)
    const double4* fbuf;
    const int* fmask;
    double2* ystage;
    int ystage_ld;
};

// ---- launch wrappers (abm_kernels.cu) ----
void launch_cells_from_colmajor(const double* cm, int n, int ncols, int ld, int has_gamma,
                                Geom* geom, Vel* vel, Phys* phys, cudaStream_t st);
void launch_cells_to_colmajor(const Geom* geom, const Vel* vel, const Phys* phys, int n, int ncols,
                              int ld, int has_gamma, double* cm, cudaStream_t st);
// 2-D layout (ABM-2d/ABM-2d-cpp/include/indices.hpp) <-> records with z = 0
void launch_cells_from_colmajor_2d(const double* cm, int n, int ncols, int ld, Geom* geom, Vel* vel, Phys* phys,
                                   cudaStream_t st);
void launch_cells_to_colmajor_2d(const Geom* geom, const Vel* vel, const Phys* phys, int n, int ncols, int ld,
                                 double* cm, cudaStream_t st);
// 2-D dE/dq (n x 4) from the pair sums (F, S): torques projected with the current n
void launch_pair_dEdq_2d(const Geom* geom, const Gen6* fcc, const Ctrl* ctrl, double* cm, int cap_cells,
                         cudaStream_t st);
// to_adhere of every CSR entry (2D/include/simulation.hpp:242-258)
void launch_adhere_flags(const Ctrl* ctrl, const int* row_ptr, const int* col, const Geom* geom, double R,
                         double Rcell, unsigned char* adhere, int cap_cells, cudaStream_t st);
void launch_gen6_to_colmajor(const Gen6* g, int n, double* cm, cudaStream_t st);

void launch_bbox(const Geom* geom, Ctrl* ctrl, Grid* grid, unsigned long long* scratch8,
                 unsigned int* counter, double edge, int cap_bins, int cap_cells, cudaStream_t st);
void launch_bin_count(const Geom* geom, const Ctrl* ctrl, const Grid* grid, int* bin_count,
                      int* key, int* slot, int cap_cells, cudaStream_t st);
void launch_bin_scatter(const Geom* geom, const Ctrl* ctrl, const int* bin_start, const int* key,
                        const int* slot, int* sorted_cell, Geom* sorted_geom, int cap_cells,
                        cudaStream_t st);
void launch_pair_build(const Grid* grid, const int* bin_start, const int* sorted_cell,
                       const Geom* sorted_geom, const Ctrl* ctrl, BuildParams bp, int* scratch,
                       int* count, int cap_bins, int num_sms, cudaStream_t st);
void launch_csr_fill(const Ctrl* ctrl, const int* row_ptr, const int* scratch, int cap_per_cell,
                     int* col, Ctrl* ctrl_w, int cap_cells, cudaStream_t st);

// exclusive scan of len (device int) entries; out has len + 1 entries, out[len] = total
void launch_scan(const int* in, const int* len, int* out, int* block_sums, int cap, cudaStream_t st);
size_t scan_block_sums_size(int cap);

// two passes: each unordered pair once from the row of its larger index, then the
// partner's share gathered from the reverse slots (jbuf, one double4 per CSR entry)
void launch_pair_force(const Geom* geom, const int* row_ptr, const int* lower_end, const int* col, const int* rev,
                       Ctrl* ctrl, ForceParams fp, const double* jkr_delta, const double* jkr_radius,
                       Gen6* fcc, double4* jbuf, int lanes, int mixed, int cap_cells, cudaStream_t st,
                       int with_gather = 1, int dims = 3);
void launch_csr_rev(const Ctrl* ctrl, const int* row_ptr, const int* col, int* lower_end, int* rev,
                    int cap_cells, cudaStream_t st);
// screened pass over every unordered pair (both shares into jbuf); with_sum also
// writes each cell's total into fcc.
void launch_pair_screened(const Geom* geom, const int* row_ptr, const int* lower_end, const int* col, const int* rev, Ctrl* ctrl, ForceParams fp, const double* jkr_delta,
                          const double* jkr_radius, Gen6* fcc, double4* jbuf, int mixed, int max_entries,
                          int cap_cells, int num_sms, cudaStream_t st, int with_sum, int dims, int tile,
                          int blocks_per_sm, const int4* pairs, int* surv, const StepParams* sp = nullptr,
                          const float* mlp_w = nullptr);
// the list of unordered pairs (i, j < i, lower entry k, partner entry rev[k]) after
// k_csr_rev, cells in `order` (null: index order): counts -> scan -> fill; uses
// `count` and `start` (cap_cells + 1) as scratch
void launch_pair_list(const Ctrl* ctrl, const int* row_ptr, const int* lower_end, const int* col, const int* rev,
                      int* count, int* start, int* block_sums, int4* pairs, int cap_cells, cudaStream_t st,
                      const int* order = nullptr);

// kind: MODE_TRIAL / MODE_RETRY / MODE_FINAL for the loop, 3 = evaluation for the API
// (writes candidates and errors without touching the controller)
// cond / use_cond: WHILE-node handle that the trial and retry attempts set to 1
// when the controller asks for another retry (only inside a CUDA graph)
void launch_attempt(int kind, Geom* geom, Vel* vel, Phys* phys, const Gen6* fcc, Ctrl* ctrl,
                    const StepParams& sp, Geom* geom_c, Vel* vel_c, Gen6* err_out, Gen6* k0buf,
                    double eval_dt, int eval_attempt, int cap_cells, cudaStream_t st,
                    unsigned long long cond = 0, int use_cond = 0, PairGather pg = PairGather{0, 0, 0, 0, 0},
                    int dims = 3, unsigned long long cond_run = 0);
// accepted proposal of the learned controller: candidate -> state (no-op otherwise)
// the attempt order of the cells (3-D): full surface solve first (made at every rebuild)
// one frame of the ring: the state after the accepted step that marked it
struct FrameInfo {
    double t;
    int iter, n, n_parents, pad;
};
// copies the cells into ring slot frames_taken % slots when a frame is due
void launch_frame_snapshot(const Geom* geom, const Vel* vel, const Phys* phys, Ctrl* ctrl, Geom* snap_geom,
                           Vel* snap_vel, Phys* snap_phys, FrameInfo* info, int slots, int cap_cells,
                           cudaStream_t st, const double* feta = nullptr, double* snap_feta = nullptr);
void launch_attempt_order(const Geom* geom, Ctrl* ctrl, const MechParams& P, int* flag, int* pos,
                          int* block_sums, int* order, int cap_cells, cudaStream_t st);
void launch_velocities(const Geom* geom, const Vel* vel, const Phys* phys, const Gen6* fcc,
                       const Ctrl* ctrl, const StepParams& sp, Gen6* v_out, int cap_cells,
                       cudaStream_t st, int dims = 3);
void launch_grow(Geom* geom, Phys* phys, const Ctrl* ctrl, double R, double dt, int cap_cells,
                 cudaStream_t st);

void launch_count_lower(const Ctrl* ctrl, const int* row_ptr, const int* col, int* cnt,
                        int cap_cells, cudaStream_t st);
void launch_table_rows(const Ctrl* ctrl, const int* row_ptr, const int* col, const int* pos,
                       const Geom* geom, double* out, int ld, int cap_cells, cudaStream_t st, int dims = 3);

// step-size network (abm_mlp.cu); weights are the flat FP32 master copy
void launch_mlp_forward(const float* master, const float* X, int n, float* Y, cudaStream_t st);
void launch_mlp_grad(const float* master, const float* X, const float* T, int n, float* G, float* loss,
                     cudaStream_t st);
void launch_mlp_train(float* master, float* m1, float* m2, float* G, const float* X, const float* T, int n,
                      int epochs, float lr, unsigned seed, float* loss_out, cudaStream_t st);
// features of the running iteration -> log row; with sp.network also the dt of the first attempt
int attempt_blocks(int cap_cells);

// division (growth.hpp:66-426), abm_divide.cu
struct DivideParams {
    double R, Rcell, Ldiv;
    double growth_mean, growth_std, daughter_length_std, angle_xy_bound, angle_z_bound;
    uint64_t seed;
    int cap_cells;
    // phenotype switching: the daughters' growth rates come from the mother's group
    // (growth.hpp:634-644), and with inherited switching one daughter of a pair may move
    // to the other group at division (switch.hpp:97-142, simulation.hpp:1650-1656)
    int group_growth;
    double gmean[2], gstd[2];
    int inherit, n_start_switch;
    double rates[4];
    double* feta;               // friction coefficient of each cell (daughters inherit it), or null
};
void launch_div_count(const Phys* phys, Ctrl* ctrl, const DivideParams& dp, int* flags,
                      unsigned long long cond, int use_cond, cudaStream_t st);
void launch_div_body_pre(Ctrl* ctrl, const int* flags, const int* rank, int* mothers, int cap_cells,
                         cudaStream_t st);
void launch_div_check(const Geom* geom, Ctrl* ctrl, const DivideParams& dp, const Grid* grid,
                      const int* bin_start, const int* sorted_cell, const Geom* sorted_geom, const int* flags,
                      const int* mothers, int* check, int* sat, cudaStream_t st);
void launch_div_tries(const Geom* geom, const Phys* phys, Ctrl* ctrl, const DivideParams& dp, const Grid* grid,
                      const int* bin_start, const int* sorted_cell, const Geom* sorted_geom, const int* flags,
                      const int* mothers, const int* check, int* sat, Geom* d1, Geom* d2, double* dlen,
                      double* dgrowth, int* ok, cudaStream_t st);
void launch_div_try_round(const Geom* geom, const Phys* phys, Ctrl* ctrl, const DivideParams& dp, const Grid* grid,
                          const int* bin_start, const int* sorted_cell, const Geom* sorted_geom, const int* flags,
                          const int* mothers, const int* check, int* sat, Geom* d1, Geom* d2, double* dlen,
                          double* dgrowth, int* ok, unsigned long long cond, cudaStream_t st);
void launch_div_commit(Geom* geom, Vel* vel, Phys* phys, Ctrl* ctrl, const DivideParams& dp, const int* mothers,
                       const Geom* d1, const Geom* d2, const double* dlen, const double* dgrowth, int* parents,
                       cudaStream_t st);

// Phenotype switching between two groups and what it drives, after each accepted step
// (abm_switch.cu): Markov switching (switch.hpp:45-95), the attribute and gamma ramps
// (simulation.hpp:1872-1957), local viscosity (simulation.hpp:1958-2020) and basal-only
// compaction (simulation.hpp:1831-1856).  Random draws: Philox, purpose SWITCH, counters
// (iteration, cell or division pair, slot).
struct SwitchParams {
    uint64_t seed;
    int mode;                   // 0 none, 1 Markov, 2 inherited at division
    int n_start;                // switching starts once the colony has this many cells
    double rates[4];            // 2 x 2, row = current group: rates (Markov) or probabilities
    double gmean[2], gstd[2];   // growth-rate distribution of each group
    double timescale;           // ramp time; 0: the attributes jump to their targets
    int n_attr;
    int attr_field[4];          // switched attributes as Phys fields: 2 eta0, 3 eta1, 4 sigma0
    double target[2][4];        // their targets in group 1 and group 2
    int gamma_ramp;             // adhesion on: gamma ramps up (group 1) or down (group 2)
    double max_gamma;
    int modulate;               // eta0 from the share of group-1 cells among the contacts
    double visc[4];             // (min, max) eta0 of group 1, then of group 2
    int max_coord;
    double R;
    int basal;                  // basal-only compaction (surface present)
    double basal_min_overlap;
};
void launch_switch_cells(Geom* geom, Phys* phys, const Ctrl* ctrl, const SwitchParams& sw, int cap_cells,
                         cudaStream_t st);
void launch_modulate_viscosity(const Geom* geom, Phys* phys, const Ctrl* ctrl, const int* row_ptr, const int* col,
                               const SwitchParams& sw, int cap_cells, cudaStream_t st);
void launch_basal_flags(const Geom* geom, const Ctrl* ctrl, const SwitchParams& sw, int* keep, int cap_cells,
                        cudaStream_t st);
void launch_basal_decide(Ctrl* ctrl, const int* keep, const int* rank, unsigned long long cond, int use_cond,
                         cudaStream_t st);
void launch_basal_compact(Geom* geom, Vel* vel, Phys* phys, Geom* geom_tmp, Vel* vel_tmp, Phys* phys_tmp,
                          Ctrl* ctrl, const int* keep, const int* rank, int cap_cells, cudaStream_t st,
                          double* feta = nullptr, double* feta_tmp = nullptr);
void launch_periodic_rebuild_cond(const Ctrl* ctrl, int every, unsigned long long cond, cudaStream_t st);

// velocity Verlet (abm_verlet.cu): one step of integration mode 0 at ctrl->dt, growth included
void launch_verlet_step(Geom* geom, Vel* vel, Phys* phys, Geom* geom_c, Vel* vel_c, double4* whalf, Ctrl* ctrl,
                        const StepParams& sp, const ForceParams& fp, const double* td, const double* tr,
                        const int4* pairs, const int* row_ptr, const int* lower_end, double4* jbuf, double4* pbuf,
                        double rho, int cap_cells, int cap_pairs, cudaStream_t st);

// friction (abm_kernels.cu): before an attempt, trial passes that run the stages of the cells
// with candidate contacts and checks that recompute the candidates' planar decisions from
// the stage states, until the decisions agree with the states (at most stages - 1 rounds)
void launch_friction_rounds(int kind, Geom* geom, Vel* vel, Phys* phys, const Gen6* fcc, Ctrl* ctrl,
                            const StepParams& sp, Geom* geom_c, Vel* vel_c, Gen6* k0buf, double eval_dt,
                            int eval_attempt, int cap_cells, cudaStream_t st, PairGather pg, const int4* pairs,
                            const int* fr_list, int* fmask, double R);

}   // namespace abm
