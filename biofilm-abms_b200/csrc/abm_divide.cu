// Division on the device: divideMaxLength + divideCells (growth.hpp:66-71, 166-426).
//
//   k_div_count    flags l > Ldiv, counts them (last block: n_divide, capacity check,
//                  sets the graph condition that enables the rest)
//   scan           exclusive scan of the flags -> mother ranks in ascending index order
//   k_div_collect  mothers[rank] = i
//   (cell list of the pre-division cells: bbox, counting sort)
//   k_div_check    room to rotate: min distance to every other cell >= 2 Rcell (minDistToCell,
//                  growth.hpp:82-117), over the bins within reach
//   10 x { k_div_try, k_div_mindist, k_div_eval }   the reference's retry loop: every try
//                  re-draws every dividing cell; the last try draws no angles
//   k_div_commit   daughter 1 keeps the mother's row, daughter 2 is appended at n + rank;
//                  IDs max_id + 2k + 1, max_id + 2k + 2; lineage appended
//   k_div_finish   n += n_divide
// Draws: Philox counters (iteration, mother rank, try, slot), slots 0-3 angles,
// 4-5 length fraction, 6-7 mother growth rate, 8-9 daughter growth rate.
#include "abm_kernels.cuh"

namespace abm {

static inline int cdiv_d(long long a, long long b) { return (int)((a + b - 1) / b); }

const int DV_T = 128;
const int DIV_TRIES = 10;

__global__ void k_div_count(const Phys* __restrict__ phys, Ctrl* ctrl, DivideParams dp, int* flags,
                            unsigned long long cond, int use_cond)
{
    __shared__ int sh_cnt;
    __shared__ bool last;
    if (threadIdx.x == 0) sh_cnt = 0;
    __syncthreads();
    const int n = ctrl->n;
    // terminate() at the top of the loop: no division and no step once n reaches the limit
    const bool halt = ctrl->halt_n > 0 && n >= ctrl->halt_n;
    int cnt = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n && !halt; i += gridDim.x * blockDim.x)
    {
        int f = phys[i].l > dp.Ldiv;          // divideMaxLength, growth.hpp:66-71
        flags[i] = f;
        cnt += f;
    }
    if (cnt) atomicAdd(&sh_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0)
    {
        if (sh_cnt) atomicAdd(&ctrl->div_count, sh_cnt);
        __threadfence();
        last = atomicAdd(&ctrl->div_blocks, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0)
    {
        __threadfence();
        int total = atomicAdd(&ctrl->div_count, 0);
        ctrl->div_count = 0;
        ctrl->div_blocks = 0u;
        if (total > 0 && n + total > dp.cap_cells)
        {
            atomicOr(&ctrl->status, (int)ST_CELL_OVERFLOW);
            total = 0;
        }
        ctrl->n_divide = total;
        ctrl->halted = halt ? 1 : 0;
        ctrl->div_done = (total == 0);
        ctrl->div_tries = 0;
        if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, total > 0 ? 1u : 0u);
    }
}

__global__ void k_div_collect(const Ctrl* ctrl, const int* flags, const int* rank, int* mothers)
{
    const int n = ctrl->n;
    if (ctrl->n_divide == 0) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flags[i]) mothers[rank[i]] = i;
}

// any other old cell j (skip == -1: none; skip_mothers: rows that now hold daughters)
// within 2 Rcell of the query segment?  Distances taken with the query as cell 1.
__device__ bool old_cells_within(const Geom& q, int self, const Grid& g, const int* __restrict__ bin_start,
                                 const int* __restrict__ sorted_cell, const Geom* __restrict__ sorted_geom,
                                 const int* flags, bool skip_mothers, double limit)
{
    const X3 rq = x3(q.rx, q.ry, q.rz), nq = x3(q.nx, q.ny, q.nz);
    const double reach = limit + q.h + g.max_half_l;
    const int rings = max(1, (int)ceil(reach * g.inv_edge));
    const int bx = min(max((int)floor((q.rx - g.x0) * g.inv_edge), 0), g.nx - 1);
    const int by = min(max((int)floor((q.ry - g.y0) * g.inv_edge), 0), g.ny - 1);
    const int bz = min(max((int)floor((q.rz - g.z0) * g.inv_edge), 0), g.nz - 1);
    for (int zz = max(bz - rings, 0); zz <= min(bz + rings, g.nz - 1); ++zz)
        for (int yy = max(by - rings, 0); yy <= min(by + rings, g.ny - 1); ++yy)
            for (int xx = max(bx - rings, 0); xx <= min(bx + rings, g.nx - 1); ++xx)
            {
                int b = (zz * g.ny + yy) * g.nx + xx;
                if (b >= g.nbins) continue;
                for (int p = bin_start[b]; p < bin_start[b + 1]; ++p)
                {
                    int j = sorted_cell[p];
                    if (j == self || (skip_mothers && flags[j])) continue;
                    Geom gj = sorted_geom[p];
                    Dist d = dist_between_cells(rq, nq, q.h, x3(gj.rx, gj.ry, gj.rz), x3(gj.nx, gj.ny, gj.nz), gj.h);
                    if (xnorm(x3(d.dx, d.dy, d.dz)) < limit) return true;
                }
            }
    return false;
}

__global__ void k_div_check(const Geom* __restrict__ geom, Ctrl* ctrl, DivideParams dp, const Grid* grid,
                            const int* bin_start, const int* sorted_cell, const Geom* sorted_geom,
                            const int* flags, const int* mothers, int* check, int* sat)
{
    const int nd = ctrl->n_divide;
    const Grid g = *grid;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nd; k += gridDim.x * blockDim.x)
    {
        int i = mothers[k];
        bool crowded = old_cells_within(load_geom(geom, i), i, g, bin_start, sorted_cell, sorted_geom, flags,
                                        false, 2 * dp.Rcell);
        check[k] = crowded ? 0 : 1;   // growth.hpp:215-226
        sat[k] = crowded ? 1 : 0;     // :231-236
    }
}

__device__ __forceinline__ double div_u(const DivideParams& dp, int iter, int k, int tr, int slot)
{
    return rng_uniform(dp.seed, RNG_PURPOSE_DIVIDE, (uint32_t)iter, (uint32_t)k, (uint32_t)tr, (uint32_t)slot);
}

// utils.hpp:791-801 (rotateXY) then :814-829 (rotateOutOfXY), in correctly rounded
// operations without FMA so daughters come out bit-identical to the CPU restatement
__device__ __forceinline__ void rotate_daughter(double ux, double uy, double uz, double txy, double tz,
                                                double& ox, double& oy, double& oz)
{
    double st, ct;
    det_sincos(txy, st, ct);
    double ax = __dadd_rn(__dadd_rn(__dmul_rn(ct, ux), __dmul_rn(-st, uy)), __dmul_rn(0.0, uz));
    double ay = __dadd_rn(__dadd_rn(__dmul_rn(st, ux), __dmul_rn(ct, uy)), __dmul_rn(0.0, uz));
    double az = __dadd_rn(__dadd_rn(__dmul_rn(0.0, ux), __dmul_rn(0.0, uy)), __dmul_rn(1.0, uz));
    // v = a x z, normalised; w = v x a
    double vx = __dsub_rn(__dmul_rn(ay, 1.0), __dmul_rn(az, 0.0));
    double vy = __dsub_rn(__dmul_rn(az, 0.0), __dmul_rn(ax, 1.0));
    double vz = __dsub_rn(__dmul_rn(ax, 0.0), __dmul_rn(ay, 0.0));
    double vn = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz)));
    vx = __ddiv_rn(vx, vn); vy = __ddiv_rn(vy, vn); vz = __ddiv_rn(vz, vn);
    double s2, c2;
    det_sincos(tz, s2, c2);
    double wx = __dsub_rn(__dmul_rn(vy, az), __dmul_rn(vz, ay));
    double wy = __dsub_rn(__dmul_rn(vz, ax), __dmul_rn(vx, az));
    double wz = __dsub_rn(__dmul_rn(vx, ay), __dmul_rn(vy, ax));
    ox = __dadd_rn(__dmul_rn(ax, c2), __dmul_rn(wx, s2));
    oy = __dadd_rn(__dmul_rn(ay, c2), __dmul_rn(wy, s2));
    oz = __dadd_rn(__dmul_rn(az, c2), __dmul_rn(wz, s2));
}

// tr_arg: the try (0 .. DIV_TRIES - 1), or -1 for the try after the ctrl->div_tries
// completed ones (the WHILE node of the iteration graph)
__global__ void k_div_try(const Geom* __restrict__ geom, const Phys* __restrict__ phys, Ctrl* ctrl,
                          DivideParams dp, const int* mothers, const int* check, int tr_arg, Geom* d1, Geom* d2,
                          double* dlen, double* dgrowth)
{
    const int nd = ctrl->n_divide;
    const int tr = tr_arg >= 0 ? tr_arg : ctrl->div_tries;
    if (nd == 0 || (tr > 0 && ctrl->div_done)) return;
    const int iter = ctrl->iter;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nd; k += gridDim.x * blockDim.x)
    {
        const int i = mothers[k];
        const Geom m = load_geom(geom, i);
        const double l = phys[i].l;
        double txy1 = 0, tz1 = 0, txy2 = 0, tz2 = 0;
        if (tr < DIV_TRIES - 1 && check[k] == 1)
        {
            const double bxy = dp.angle_xy_bound, bz = dp.angle_z_bound;
            txy1 = __dadd_rn(-bxy, __dmul_rn(__dmul_rn(2.0, bxy), div_u(dp, iter, k, tr, 0)));
            tz1 = __dadd_rn(-bz, __dmul_rn(__dmul_rn(2.0, bz), div_u(dp, iter, k, tr, 1)));
            txy2 = __dadd_rn(-bxy, __dmul_rn(__dmul_rn(2.0, bxy), div_u(dp, iter, k, tr, 2)));
            tz2 = __dadd_rn(-bz, __dmul_rn(__dmul_rn(2.0, bz), div_u(dp, iter, k, tr, 3)));
        }
        Geom a = m, b = m;
        rotate_daughter(m.nx, m.ny, m.nz, txy1, tz1, a.nx, a.ny, a.nz);
        rotate_daughter(m.nx, m.ny, m.nz, txy2, tz2, b.nx, b.ny, b.nz);
        // growth.hpp:311-348: lengths M (L - 2R), (1 - M)(L - 2R) and centres either side of
        // the division point (correctly rounded operations, as the CPU restatement)
        double r = __dadd_rn(0.5, __dmul_rn(dp.daughter_length_std,
                                            std_normal(div_u(dp, iter, k, tr, 4), div_u(dp, iter, k, tr, 5))));
        double M = r < 0 ? 0.0 : (r > 1 ? 1.0 : r);
        double Ld = __dsub_rn(l, __dmul_rn(2.0, dp.R));
        double L1 = __dmul_rn(M, Ld), L2 = __dmul_rn(__dsub_rn(1.0, M), Ld);
        double dv = __dadd_rn(__dadd_rn(-m.h, L1), dp.R);
        double del1 = __dadd_rn(__ddiv_rn(L1, 2.0), dp.R), del2 = __dadd_rn(__ddiv_rn(L2, 2.0), dp.R);
        double f1 = __dsub_rn(dv, del1), f2 = __dadd_rn(dv, del2);
        a.rx = __dadd_rn(m.rx, __dmul_rn(f1, a.nx)); a.ry = __dadd_rn(m.ry, __dmul_rn(f1, a.ny));
        a.rz = __dadd_rn(m.rz, __dmul_rn(f1, a.nz));
        b.rx = __dadd_rn(m.rx, __dmul_rn(f2, b.nx)); b.ry = __dadd_rn(m.ry, __dmul_rn(f2, b.ny));
        b.rz = __dadd_rn(m.rz, __dmul_rn(f2, b.nz));
        a.h = __ddiv_rn(L1, 2.0); b.h = __ddiv_rn(L2, 2.0);
        d1[k] = a; d2[k] = b;
        dlen[2 * k] = L1; dlen[2 * k + 1] = L2;
        // with switching, the distribution of the mother's group (growth.hpp:634-644)
        double gmean = dp.growth_mean, gstd = dp.growth_std;
        if (dp.group_growth)
        {
            const int g0 = (int)phys[i].group == 1 ? 0 : 1;
            gmean = dp.gmean[g0]; gstd = dp.gstd[g0];
        }
        dgrowth[2 * k] = __dadd_rn(gmean, __dmul_rn(gstd,
                                   std_normal(div_u(dp, iter, k, tr, 6), div_u(dp, iter, k, tr, 7))));
        dgrowth[2 * k + 1] = __dadd_rn(gmean, __dmul_rn(gstd,
                                       std_normal(div_u(dp, iter, k, tr, 8), div_u(dp, iter, k, tr, 9))));
    }
}

// min distance of each daughter to the new population >= 2 Rcell?  (growth.hpp:366-398)
__global__ void k_div_mindist(Ctrl* ctrl, DivideParams dp, const Grid* grid, const int* bin_start,
                              const int* sorted_cell, const Geom* sorted_geom, const int* flags,
                              const int* mothers, const int* check, int tr_arg, const Geom* d1, const Geom* d2,
                              int* ok)
{
    const int nd = ctrl->n_divide;
    const int tr = tr_arg >= 0 ? tr_arg : ctrl->div_tries;
    if (nd == 0 || (tr > 0 && ctrl->div_done)) return;
    const Grid g = *grid;
    const double limit = 2 * dp.Rcell;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 2 * nd; q += gridDim.x * blockDim.x)
    {
        const int k = q >> 1, which = q & 1;
        if (check[k] != 1) { ok[q] = 0; continue; }
        const Geom dq = which ? d2[k] : d1[k];
        bool close = old_cells_within(dq, mothers[k], g, bin_start, sorted_cell, sorted_geom, flags, true, limit);
        const X3 rq = x3(dq.rx, dq.ry, dq.rz), nq = x3(dq.nx, dq.ny, dq.nz);
        for (int o = 0; o < 2 * nd && !close; ++o)
        {
            if (o == q) continue;
            const Geom go = (o & 1) ? d2[o >> 1] : d1[o >> 1];
            Dist d = dist_between_cells(rq, nq, dq.h, x3(go.rx, go.ry, go.rz), x3(go.nx, go.ny, go.nz), go.h);
            if (xnorm(x3(d.dx, d.dy, d.dz)) < limit) close = true;
        }
        ok[q] = close ? 0 : 1;
    }
}

// use_cond: `cond` is the handle of the WHILE node around the tries, continued while
// a dividing cell still misses the distance criterion and tries are left
__global__ void k_div_eval(Ctrl* ctrl, const int* check, const int* ok, int* sat, int tr_arg,
                           unsigned long long cond, int use_cond)
{
    __shared__ int sh;
    __shared__ bool last;
    const int nd = ctrl->n_divide;
    const int tr = tr_arg >= 0 ? tr_arg : ctrl->div_tries;
    if (nd == 0 || (tr > 0 && ctrl->div_done))
    {
        if (use_cond && blockIdx.x == 0 && threadIdx.x == 0)
            cudaGraphSetConditional((cudaGraphConditionalHandle)cond, 0u);
        return;
    }
    if (threadIdx.x == 0) sh = 0;
    __syncthreads();
    int c = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nd; k += gridDim.x * blockDim.x)
    {
        if (check[k] == 1 && ok[2 * k] && ok[2 * k + 1]) sat[k] = 1;
        c += sat[k];
    }
    if (c) atomicAdd(&sh, c);
    __syncthreads();
    if (threadIdx.x == 0)
    {
        if (sh) atomicAdd(&ctrl->div_count, sh);
        __threadfence();
        last = atomicAdd(&ctrl->div_blocks, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0)
    {
        __threadfence();
        int total = atomicAdd(&ctrl->div_count, 0);
        ctrl->div_count = 0;
        ctrl->div_blocks = 0u;
        ctrl->div_tries = tr + 1;
        // while (ntries == 0 || (ntries < 10 && satisfied < n_divide))  (growth.hpp:252)
        ctrl->div_done = (total >= nd) || (tr + 1 >= DIV_TRIES);
        if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, ctrl->div_done ? 0u : 1u);
    }
}

// switch.hpp:97-142 (switchGroupsInherit) for division pair k, the daughters in the
// mother's row (p1) and the appended row (p2), both of the mother's group g: with
// probability 1 - P(g, g), one of the two, chosen by a second uniform, moves to the other
// group and draws that group's growth rate.  Draws: purpose SWITCH, counters (iteration,
// pair, slot 4 / 5 / 6-7).
__device__ __forceinline__ void inherit_switch(const DivideParams& dp, int iter, int k, Phys& p1, Phys& p2)
{
    const int g = (int)p1.group - 1;
    if (g != 0 && g != 1) return;
    auto u = [&](int slot) {
        return rng_uniform(dp.seed, RNG_PURPOSE_SWITCH, (uint32_t)iter, (uint32_t)k, (uint32_t)slot, 0u);
    };
    const double r = u(4);
    double total = dp.rates[g * 2 + g];
    if (!(r > total)) return;
    for (int j = 0; j < 2; ++j)
    {
        if (j == g) continue;
        const double prob = dp.rates[g * 2 + j];
        if (r > total && r < __dadd_rn(total, prob))
        {
            Phys& w = u(5) < 0.5 ? p1 : p2;
            w.group = j + 1;
            w.growth = __dadd_rn(dp.gmean[j], __dmul_rn(dp.gstd[j], std_normal(u(6), u(7))));
            return;
        }
        total = __dadd_rn(total, prob);
    }
}

__global__ void k_div_commit(Geom* geom, Vel* vel, Phys* phys, const Ctrl* ctrl, DivideParams dp, const int* mothers,
                             const Geom* d1, const Geom* d2, const double* dlen, const double* dgrowth,
                             int* parents)
{
    const int nd = ctrl->n_divide;
    const int n = ctrl->n;
    const int np = ctrl->n_parents;
    const double t = ctrl->t;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nd; k += gridDim.x * blockDim.x)
    {
        const int i = mothers[k];
        const Phys pm = phys[i];
        const Vel vm = vel[i];
        const int parent_id = (int)pm.id;
        const int max_id = np - 1;
        Geom a = d1[k], b = d2[k];
        Phys p1 = pm, p2 = pm;
        p1.l = dlen[2 * k]; p2.l = dlen[2 * k + 1];
        p1.t0 = t; p2.t0 = t;
        p1.growth = dgrowth[2 * k]; p2.growth = dgrowth[2 * k + 1];
        p1.id = max_id + (2 * k + 1); p2.id = max_id + (2 * k + 2);   // growth.hpp:407-418
        if (dp.inherit && n + nd >= dp.n_start_switch) inherit_switch(dp, ctrl->iter, k, p1, p2);
        geom[i] = a; phys[i] = p1;
        geom[n + k] = b; phys[n + k] = p2; vel[n + k] = vm;
        if (dp.feta) dp.feta[n + k] = dp.feta[i];
        parents[np + 2 * k] = parent_id;
        parents[np + 2 * k + 1] = parent_id;
    }
}

__global__ void k_div_finish(Ctrl* ctrl)
{
    const int nd = ctrl->n_divide;
    if (nd == 0) return;
    ctrl->n += nd;
    ctrl->n_parents += 2 * nd;
    ctrl->divisions += nd;
    ctrl->div_events += 1;
    ctrl->last_div_tries = ctrl->div_tries;
    ctrl->n_divide = 0;
    ctrl->screen_valid = 0;            // new cells: the active pair list is stale
}

void launch_div_count(const Phys* phys, Ctrl* ctrl, const DivideParams& dp, int* flags,
                      unsigned long long cond, int use_cond, cudaStream_t st)
{
    int blocks = max(min(cdiv_d(dp.cap_cells, 256), 296), 1);
    k_div_count<<<blocks, 256, 0, st>>>(phys, ctrl, dp, flags, cond, use_cond);
}

void launch_div_body_pre(Ctrl* ctrl, const int* flags, const int* rank, int* mothers, int cap_cells,
                         cudaStream_t st)
{
    k_div_collect<<<max(cdiv_d(cap_cells, 256), 1), 256, 0, st>>>(ctrl, flags, rank, mothers);
}

void launch_div_check(const Geom* geom, Ctrl* ctrl, const DivideParams& dp, const Grid* grid,
                      const int* bin_start, const int* sorted_cell, const Geom* sorted_geom, const int* flags,
                      const int* mothers, int* check, int* sat, cudaStream_t st)
{
    k_div_check<<<max(cdiv_d(dp.cap_cells, DV_T), 1), DV_T, 0, st>>>(geom, ctrl, dp, grid, bin_start, sorted_cell,
                                                                   sorted_geom, flags, mothers, check, sat);
}

void launch_div_tries(const Geom* geom, const Phys* phys, Ctrl* ctrl, const DivideParams& dp, const Grid* grid,
                      const int* bin_start, const int* sorted_cell, const Geom* sorted_geom, const int* flags,
                      const int* mothers, const int* check, int* sat, Geom* d1, Geom* d2, double* dlen,
                      double* dgrowth, int* ok, cudaStream_t st)
{
    const int b1 = max(cdiv_d(dp.cap_cells, DV_T), 1), b2 = max(cdiv_d(2LL * dp.cap_cells, DV_T), 1);
    for (int tr = 0; tr < DIV_TRIES; ++tr)
    {
        k_div_try<<<b1, DV_T, 0, st>>>(geom, phys, ctrl, dp, mothers, check, tr, d1, d2, dlen, dgrowth);
        k_div_mindist<<<b2, DV_T, 0, st>>>(ctrl, dp, grid, bin_start, sorted_cell, sorted_geom, flags, mothers,
                                          check, tr, d1, d2, ok);
        k_div_eval<<<b1, DV_T, 0, st>>>(ctrl, check, ok, sat, tr, 0, 0);
    }
}

// one try of the body of the WHILE node (the try index from ctrl->div_tries)
void launch_div_try_round(const Geom* geom, const Phys* phys, Ctrl* ctrl, const DivideParams& dp, const Grid* grid,
                          const int* bin_start, const int* sorted_cell, const Geom* sorted_geom, const int* flags,
                          const int* mothers, const int* check, int* sat, Geom* d1, Geom* d2, double* dlen,
                          double* dgrowth, int* ok, unsigned long long cond, cudaStream_t st)
{
    const int b1 = max(cdiv_d(dp.cap_cells, DV_T), 1), b2 = max(cdiv_d(2LL * dp.cap_cells, DV_T), 1);
    k_div_try<<<b1, DV_T, 0, st>>>(geom, phys, ctrl, dp, mothers, check, -1, d1, d2, dlen, dgrowth);
    k_div_mindist<<<b2, DV_T, 0, st>>>(ctrl, dp, grid, bin_start, sorted_cell, sorted_geom, flags, mothers,
                                      check, -1, d1, d2, ok);
    k_div_eval<<<b1, DV_T, 0, st>>>(ctrl, check, ok, sat, -1, cond, 1);
}

void launch_div_commit(Geom* geom, Vel* vel, Phys* phys, Ctrl* ctrl, const DivideParams& dp, const int* mothers,
                       const Geom* d1, const Geom* d2, const double* dlen, const double* dgrowth, int* parents,
                       cudaStream_t st)
{
    k_div_commit<<<max(cdiv_d(dp.cap_cells, DV_T), 1), DV_T, 0, st>>>(geom, vel, phys, ctrl, dp, mothers, d1, d2,
                                                                     dlen, dgrowth, parents);
    k_div_finish<<<1, 1, 0, st>>>(ctrl);
}

}   // namespace abm
