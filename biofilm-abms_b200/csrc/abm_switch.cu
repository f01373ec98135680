// Phenotype switching between two groups and what it drives, run after each accepted
// step of the loop (kmnam/biofilm-ABMs, ABM-3d/ABM-3d-cpp/include):
//   * Markov switching (switch.hpp:45-95): each cell of group g moves to group j when a
//     uniform r falls in [sum of the earlier probabilities, + dt rate(g, j)), and then
//     draws j's growth rate;
//   * the attribute ramps (simulation.hpp:1872-1938): each switched attribute moves toward
//     its group's target at |target1 - target2| / timescale per unit time, stopping there;
//   * the gamma ramp (simulation.hpp:1940-1957): gamma rises toward max_gamma in group 1,
//     falls toward 0 in group 2, at max_gamma / timescale;
//   * local viscosity (simulation.hpp:1958-2020): eta0 interpolates between the group's
//     limits by the share of group-1 cells among the contacts (distance < 2R);
//   * basal-only compaction (simulation.hpp:1831-1856): with the surface present only
//     cells whose deepest overlap R - rz + half_l nz exceeds a threshold stay, in order.
// The random draws use the counter-based Philox policy of the division and noise
// kernels (purpose SWITCH, counters iteration, cell, slot), so the device takes the same
// decisions as a sequential CPU loop with the same policy, cell for cell.  Every
// floating-point operation is a correctly rounded intrinsic in the CPU loop's order.
#include "abm_kernels.cuh"

namespace abm {

const int SW_T = 256;

static inline int cdiv_s(int a, int b) { return (a + b - 1) / b; }

__device__ __forceinline__ double sw_uniform(const SwitchParams& sw, int iter, int k, int slot)
{
    return rng_uniform(sw.seed, RNG_PURPOSE_SWITCH, (uint32_t)iter, (uint32_t)k, (uint32_t)slot, 0u);
}

// growth rate drawn from group g0's distribution (0-based) at slots (slot, slot + 1)
__device__ __forceinline__ double sw_growth(const SwitchParams& sw, int g0, int iter, int k, int slot)
{
    return __dadd_rn(sw.gmean[g0], __dmul_rn(sw.gstd[g0], std_normal(sw_uniform(sw, iter, k, slot),
                                                                     sw_uniform(sw, iter, k, slot + 1))));
}

// dt of the step just accepted (the ring's newest entry)
__device__ __forceinline__ double accepted_dt(const Ctrl* c)
{
    return c->hist_dt[(c->hist_pos + HIST - 1) % HIST];
}

// Markov switching, then the attribute and gamma ramps, one cell per thread: each cell's
// updates read only its own state and draws
__global__ void k_switch_cells(Geom* geom, Phys* phys, const Ctrl* ctrl, SwitchParams sw)
{
    if (ctrl->halted) return;
    const int n = ctrl->n;
    const int iter = ctrl->iter;
    const double dt = accepted_dt(ctrl);
    const bool markov = sw.mode == 1 && n >= sw.n_start;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        double* ph = reinterpret_cast<double*>(phys + i);
        Phys p = phys[i];
        bool dirty = false;
        const int g = (int)p.group - 1;
        if (markov && (g == 0 || g == 1))
        {
            const double r = sw_uniform(sw, iter, i, 0);
            double total = 0;
            for (int j = 0; j < 2; ++j)
            {
                if (j == g) continue;
                const double prob = __dmul_rn(dt, sw.rates[g * 2 + j]);
                if (r > total && r < __dadd_rn(total, prob))
                {
                    p.group = j + 1;
                    p.growth = sw_growth(sw, j, iter, i, 2);
                    dirty = true;
                    break;
                }
                total = __dadd_rn(total, prob);
            }
        }
        if (dirty) { phys[i].group = p.group; phys[i].growth = p.growth; }
        const bool g1 = (int)p.group == 1;
        for (int k = 0; k < sw.n_attr; ++k)
        {
            const double t1 = sw.target[0][k], t2 = sw.target[1][k];
            const double own = g1 ? t1 : t2, other = g1 ? t2 : t1;
            double v = ph[sw.attr_field[k]];
            const double v0 = v;
            if (sw.timescale == 0) { if (v != own) v = own; }
            else
            {
                const double step = __dmul_rn(__ddiv_rn(fabs(__dsub_rn(t1, t2)), sw.timescale), dt);
                if (own > other && v < own) { v = __dadd_rn(v, step); if (v > own) v = own; }
                else if (own < other && v > own) { v = __dsub_rn(v, step); if (v < own) v = own; }
                else if (t1 == t2 && v != own) v = own;
            }
            if (v != v0) ph[sw.attr_field[k]] = v;
        }
        if (sw.gamma_ramp)
        {
            double gm = geom[i].gamma;
            const double g0 = gm;
            if (sw.timescale == 0)
            {
                // an infinite rate: the ramp lands on its bound at once
                if (g1) { if (gm < sw.max_gamma) gm = sw.max_gamma; }
                else if (gm > 0) gm = 0;
            }
            else
            {
                const double step = __dmul_rn(__ddiv_rn(sw.max_gamma, sw.timescale), dt);
                if (g1) { if (gm < sw.max_gamma) { gm = __dadd_rn(gm, step); if (gm > sw.max_gamma) gm = sw.max_gamma; } }
                else if (gm > 0) { gm = __dsub_rn(gm, step); if (gm < 0) gm = 0; }
            }
            if (gm != g0) geom[i].gamma = gm;
        }
    }
}

// local viscosity, one cell per thread over its neighbor row: a contact is a neighbor
// at distance < 2R, the distance evaluated with the larger index as cell 1 as the
// neighbor list stores it, so both cells of a pair count the same contact
__global__ void k_modulate_viscosity(const Geom* __restrict__ geom, Phys* phys, const Ctrl* ctrl,
                                     const int* __restrict__ row_ptr, const int* __restrict__ col, SwitchParams sw)
{
    if (ctrl->halted) return;
    const int n = ctrl->n;
    const double lim = 2 * sw.R;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        int total = 0, g1 = 0;
        const Geom gi = load_geom(geom, i);
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
        {
            const int j = col[k];
            const Geom gj = load_geom(geom, j);
            const Dist d = j < i ? dist_geom(gi, gj) : dist_geom(gj, gi);
            const double nrm = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d.dx, d.dx), __dmul_rn(d.dy, d.dy)),
                                                    __dmul_rn(d.dz, d.dz)));
            if (nrm < lim)
            {
                total += 1;
                if ((int)phys[j].group == 1) g1 += 1;
            }
        }
        const int g = (int)phys[i].group - 1;
        if (g != 0 && g != 1) continue;           // groups are 1 and 2
        const double vmin = sw.visc[g * 2], vmax = sw.visc[g * 2 + 1];
        double eta0;
        if (g1 >= sw.max_coord) eta0 = vmax;
        else
        {
            const double ratio = __ddiv_rn((double)g1, (double)max(total, sw.max_coord));
            eta0 = __dadd_rn(vmin, __dmul_rn(ratio, __dsub_rn(vmax, vmin)));
        }
        phys[i].eta0 = eta0;
    }
}

// basal-only: keep[i] = 1 when the deepest overlap exceeds the threshold
__global__ void k_basal_flags(const Geom* __restrict__ geom, const Ctrl* ctrl, SwitchParams sw, int* keep)
{
    if (ctrl->halted) return;
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const Geom g = load_geom(geom, i);
        keep[i] = __dadd_rn(__dsub_rn(sw.R, g.rz), __dmul_rn(g.h, g.nz)) > sw.basal_min_overlap ? 1 : 0;
    }
}

// the kept count from the exclusive scan; with use_cond the IF node around the
// compaction runs only when a cell is dropped
__global__ void k_basal_decide(Ctrl* ctrl, const int* keep, const int* rank, unsigned long long cond, int use_cond)
{
    const int n = ctrl->n;
    const int kept = (ctrl->halted || n == 0) ? n : rank[n - 1] + keep[n - 1];
    ctrl->n_keep = kept;
    if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, kept < n ? 1u : 0u);
}

__global__ void k_basal_scatter(const Geom* geom, const Vel* vel, const Phys* phys, Geom* geom_tmp, Vel* vel_tmp,
                                Phys* phys_tmp, const Ctrl* ctrl, const int* keep, const int* rank,
                                const double* feta, double* feta_tmp)
{
    const int n = ctrl->n;
    if (ctrl->n_keep >= n) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (keep[i])
        {
            const int r = rank[i];
            geom_tmp[r] = geom[i]; vel_tmp[r] = vel[i]; phys_tmp[r] = phys[i];
            if (feta) feta_tmp[r] = feta[i];
        }
}

__global__ void k_basal_gather(Geom* geom, Vel* vel, Phys* phys, const Geom* geom_tmp, const Vel* vel_tmp,
                               const Phys* phys_tmp, const Ctrl* ctrl, double* feta, const double* feta_tmp)
{
    const int m = ctrl->n_keep;
    if (m >= ctrl->n) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    {
        geom[i] = geom_tmp[i]; vel[i] = vel_tmp[i]; phys[i] = phys_tmp[i];
        if (feta) feta[i] = feta_tmp[i];
    }
}

__global__ void k_basal_commit(Ctrl* ctrl)
{
    const int m = ctrl->n_keep;
    if (m >= ctrl->n) return;
    ctrl->basal_dropped += ctrl->n - m;
    ctrl->n = m;
    ctrl->screen_valid = 0;          // the active pair list names the old rows
    ctrl->n_order = 0;
}

// IF node of the periodic neighbor rebuild (simulation.hpp:1848-1856): the iteration
// counter, advanced by the accepted step, is a multiple of `every`
__global__ void k_periodic_cond(const Ctrl* ctrl, int every, unsigned long long cond)
{
    const bool due = !ctrl->halted && ctrl->iter % every == 0;
    cudaGraphSetConditional((cudaGraphConditionalHandle)cond, due ? 1u : 0u);
}

static int sw_blocks(int cap_cells) { return max(min(cdiv_s(cap_cells, SW_T), 148 * 8), 1); }

void launch_switch_cells(Geom* geom, Phys* phys, const Ctrl* ctrl, const SwitchParams& sw, int cap_cells,
                         cudaStream_t st)
{
    k_switch_cells<<<sw_blocks(cap_cells), SW_T, 0, st>>>(geom, phys, ctrl, sw);
}

void launch_modulate_viscosity(const Geom* geom, Phys* phys, const Ctrl* ctrl, const int* row_ptr, const int* col,
                               const SwitchParams& sw, int cap_cells, cudaStream_t st)
{
    k_modulate_viscosity<<<sw_blocks(cap_cells), SW_T, 0, st>>>(geom, phys, ctrl, row_ptr, col, sw);
}

void launch_basal_flags(const Geom* geom, const Ctrl* ctrl, const SwitchParams& sw, int* keep, int cap_cells,
                        cudaStream_t st)
{
    k_basal_flags<<<sw_blocks(cap_cells), SW_T, 0, st>>>(geom, ctrl, sw, keep);
}

void launch_basal_decide(Ctrl* ctrl, const int* keep, const int* rank, unsigned long long cond, int use_cond,
                         cudaStream_t st)
{
    k_basal_decide<<<1, 1, 0, st>>>(ctrl, keep, rank, cond, use_cond);
}

void launch_basal_compact(Geom* geom, Vel* vel, Phys* phys, Geom* geom_tmp, Vel* vel_tmp, Phys* phys_tmp,
                          Ctrl* ctrl, const int* keep, const int* rank, int cap_cells, cudaStream_t st,
                          double* feta, double* feta_tmp)
{
    const int b = sw_blocks(cap_cells);
    k_basal_scatter<<<b, SW_T, 0, st>>>(geom, vel, phys, geom_tmp, vel_tmp, phys_tmp, ctrl, keep, rank, feta,
                                        feta_tmp);
    k_basal_gather<<<b, SW_T, 0, st>>>(geom, vel, phys, geom_tmp, vel_tmp, phys_tmp, ctrl, feta, feta_tmp);
    k_basal_commit<<<1, 1, 0, st>>>(ctrl);
}

void launch_periodic_rebuild_cond(const Ctrl* ctrl, int every, unsigned long long cond, cudaStream_t st)
{
    k_periodic_cond<<<1, 1, 0, st>>>(ctrl, every, cond);
}

}   // namespace abm
