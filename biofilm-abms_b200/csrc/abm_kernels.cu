// CUDA kernels of the B200 mechanics step (sm_100a).
//
//   cell list      k_bbox -> k_bin_count -> scan -> k_bin_scatter        (uniform grid,
//                  counting sort by bin)
//   pair set       k_pair_build -> scan -> k_csr_fill -> k_csr_rev      (getCellNeighbors,
//                  mechanics.hpp:520-593; CSR rows sorted by neighbor index), then the
//                  pair records in bin order and the attempt order
//   pair force     k_pair_pass<MIXED, DIM>                              (cellCellInteractionForces,
//                  mechanics.hpp:1209-1659; one record per unordered pair, screened
//                  against an active list with a skin, both shares per pair; the last
//                  block makes the step-size proposal of the learned controller)
//                  k_pair_force<G> serves the no-alloc entry point (G lanes per cell)
//   RK attempt     k_attempt<S, KIND>                                   (stepRungeKuttaAdaptive,
//                  mechanics.hpp:2406-2612; all stages of a cell in registers, the error
//                  norm reduced in the same kernel, the step-size controller of
//                  simulation.hpp:1690-1769 run by the last block to finish)
#include <cstdio>
#include "abm_kernels.cuh"
#include "abm_pair.cuh"
#include "abm_propose.cuh"

namespace abm {

static inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// Order-preserving double <-> uint64 maps for atomic min/max
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ord_enc(double x)
{
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_dec(unsigned long long u)
{
    u = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
    return __longlong_as_double((long long)u);
}

// ---------------------------------------------------------------------------
// Column-major cell arrays <-> device records
// ---------------------------------------------------------------------------
__global__ void k_cells_from_colmajor(const double* __restrict__ cm, int n, int ncols, int ld,
                                      int has_gamma, Geom* geom, Vel* vel, Phys* phys)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    auto c = [&](int col) { return cm[(size_t)col * ld + i]; };
    Geom g;
    g.rx = c(1); g.ry = c(2); g.rz = c(3); g.h = c(14);
    g.nx = c(4); g.ny = c(5); g.nz = c(6); g.gamma = has_gamma ? c(21) : 0.0;
    geom[i] = g;
    Vel v;
    for (int k = 0; k < 6; ++k) v.v[k] = c(7 + k);
    vel[i] = v;
    Phys p;
    p.l = c(13); p.growth = c(16); p.eta0 = c(17); p.eta1 = c(18); p.sigma0 = c(19);
    p.t0 = c(15); p.id = c(0); p.group = c(20);
    phys[i] = p;
}

__global__ void k_cells_to_colmajor(const Geom* __restrict__ geom, const Vel* __restrict__ vel,
                                    const Phys* __restrict__ phys, int n, int ncols, int ld,
                                    int has_gamma, double* cm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Geom g = geom[i]; Vel v = vel[i]; Phys p = phys[i];
    auto w = [&](int col, double x) { cm[(size_t)col * ld + i] = x; };
    w(0, p.id); w(1, g.rx); w(2, g.ry); w(3, g.rz); w(4, g.nx); w(5, g.ny); w(6, g.nz);
    for (int k = 0; k < 6; ++k) w(7 + k, v.v[k]);
    w(13, p.l); w(14, g.h); w(15, p.t0); w(16, p.growth); w(17, p.eta0); w(18, p.eta1);
    w(19, p.sigma0); w(20, p.group);
    if (has_gamma && ncols > 21) w(21, g.gamma);
}

__global__ void k_gen6_to_colmajor(const Gen6* __restrict__ g, int n, double* cm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Gen6 v = g[i];
    for (int k = 0; k < 6; ++k) cm[(size_t)k * n + i] = v.f[k];
}

// 2-D layout (ABM-2d/ABM-2d-cpp/include/indices.hpp:17-41): id, r(2), n(2), dr(2), dn(2),
// l, half_l, t0, growth, eta0, eta1, maxeta1, group; the records hold z = nz = 0 and
// maxeta1 in the sigma0 slot
__global__ void k_cells_from_colmajor_2d(const double* __restrict__ cm, int n, int ld, Geom* geom, Vel* vel,
                                         Phys* phys)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    auto c = [&](int col) { return cm[(size_t)col * ld + i]; };
    Geom g;
    g.rx = c(1); g.ry = c(2); g.rz = 0.0; g.h = c(10);
    g.nx = c(3); g.ny = c(4); g.nz = 0.0; g.gamma = 0.0;
    geom[i] = g;
    Vel v;
    v.v[0] = c(5); v.v[1] = c(6); v.v[2] = 0.0; v.v[3] = c(7); v.v[4] = c(8); v.v[5] = 0.0;
    vel[i] = v;
    Phys p;
    p.l = c(9); p.t0 = c(11); p.growth = c(12); p.eta0 = c(13); p.eta1 = c(14); p.sigma0 = c(15);
    p.id = c(0); p.group = c(16);
    phys[i] = p;
}

__global__ void k_cells_to_colmajor_2d(const Geom* __restrict__ geom, const Vel* __restrict__ vel,
                                       const Phys* __restrict__ phys, int n, int ld, double* cm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Geom g = geom[i]; Vel v = vel[i]; Phys p = phys[i];
    auto w = [&](int col, double x) { cm[(size_t)col * ld + i] = x; };
    w(0, p.id); w(1, g.rx); w(2, g.ry); w(3, g.nx); w(4, g.ny);
    w(5, v.v[0]); w(6, v.v[1]); w(7, v.v[3]); w(8, v.v[4]);
    w(9, p.l); w(10, g.h); w(11, p.t0); w(12, p.growth); w(13, p.eta0); w(14, p.eta1); w(15, p.sigma0);
    w(16, p.group);
}

void launch_cells_from_colmajor_2d(const double* cm, int n, int ncols, int ld, Geom* geom, Vel* vel, Phys* phys,
                                   cudaStream_t st)
{
    if (n <= 0) return;
    k_cells_from_colmajor_2d<<<cdiv(n, 256), 256, 0, st>>>(cm, n, ld, geom, vel, phys);
}

void launch_cells_to_colmajor_2d(const Geom* geom, const Vel* vel, const Phys* phys, int n, int ncols, int ld,
                                 double* cm, cudaStream_t st)
{
    if (n <= 0) return;
    k_cells_to_colmajor_2d<<<cdiv(n, 256), 256, 0, st>>>(geom, vel, phys, n, ld, cm);
}

void launch_cells_from_colmajor(const double* cm, int n, int ncols, int ld, int has_gamma,
                                Geom* geom, Vel* vel, Phys* phys, cudaStream_t st)
{
    if (n <= 0) return;
    k_cells_from_colmajor<<<cdiv(n, 256), 256, 0, st>>>(cm, n, ncols, ld, has_gamma, geom, vel, phys);
}
void launch_cells_to_colmajor(const Geom* geom, const Vel* vel, const Phys* phys, int n, int ncols,
                              int ld, int has_gamma, double* cm, cudaStream_t st)
{
    if (n <= 0) return;
    k_cells_to_colmajor<<<cdiv(n, 256), 256, 0, st>>>(geom, vel, phys, n, ncols, ld, has_gamma, cm);
}
void launch_gen6_to_colmajor(const Gen6* g, int n, double* cm, cudaStream_t st)
{
    if (n <= 0) return;
    k_gen6_to_colmajor<<<cdiv(n, 256), 256, 0, st>>>(g, n, cm);
}

// ---------------------------------------------------------------------------
// Block reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// Cell list: bounding box -> grid (last block), counting sort by bin
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_bbox(const Geom* __restrict__ geom, Ctrl* ctrl, Grid* grid,
                                              unsigned long long* acc, unsigned int* counter,
                                              double edge, int cap_bins)
{
    __shared__ double sh[7][8];
    __shared__ bool last;
    const int n = ctrl->n;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300}, mh = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        Geom g = load_geom(geom, i);
        mn[0] = fmin(mn[0], g.rx); mn[1] = fmin(mn[1], g.ry); mn[2] = fmin(mn[2], g.rz);
        mx[0] = fmax(mx[0], g.rx); mx[1] = fmax(mx[1], g.ry); mx[2] = fmax(mx[2], g.rz);
        mh = fmax(mh, g.h);
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double v[7] = {mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], mh};
    for (int k = 0; k < 3; ++k) v[k] = warp_min(v[k]);
    for (int k = 3; k < 7; ++k) v[k] = warp_max(v[k]);
    if (lane == 0) for (int k = 0; k < 7; ++k) sh[k][wid] = v[k];
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
        {
            for (int k = 0; k < 3; ++k) v[k] = fmin(v[k], sh[k][w]);
            for (int k = 3; k < 7; ++k) v[k] = fmax(v[k], sh[k][w]);
        }
        for (int k = 0; k < 3; ++k) atomicMin(&acc[k], ord_enc(v[k]));
        for (int k = 3; k < 7; ++k) atomicMax(&acc[k], ord_enc(v[k]));
        __threadfence();
        unsigned int done = atomicAdd(counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0)
    {
        __threadfence();
        double lo[3], hi[3];
        for (int k = 0; k < 3; ++k)
        {
            lo[k] = ord_dec(atomicAdd(&acc[k], 0ull));
            hi[k] = ord_dec(atomicAdd(&acc[3 + k], 0ull));
        }
        double maxh = ord_dec(atomicAdd(&acc[6], 0ull));
        if (n <= 0) { for (int k = 0; k < 3; ++k) { lo[k] = 0; hi[k] = 0; } maxh = 0; }
        // fmin / fmax skip NaN coordinates; an axis without any finite one spans [0, 0], and
        // an infinite extent, or one no grid of cap_bins bins can hold, is an overflow
        bool bad = false;
        for (int k = 0; k < 3; ++k)
        {
            if (!(lo[k] <= hi[k])) { lo[k] = 0; hi[k] = 0; }
            if (!(hi[k] - lo[k] < 1e290)) bad = true;
        }
        double e = edge;
        double nb[3] = {1.0, 1.0, 1.0};
        for (int tries = 0; tries < 64 && !bad; ++tries)
        {
            for (int k = 0; k < 3; ++k) nb[k] = floor((hi[k] - lo[k]) / e) + 1;
            if (nb[0] * nb[1] * nb[2] <= (double)cap_bins) break;
            e *= 1.5;
        }
        if (bad || !(nb[0] * nb[1] * nb[2] <= (double)cap_bins))
        {
            // one bin: every later kernel stays in bounds, the pair build skips its work
            // (the status is set) and the host reports the overflow
            atomicOr(&ctrl->status, (int)ST_BIN_OVERFLOW);
            for (int k = 0; k < 3; ++k) { nb[k] = 1.0; lo[k] = 0.0; }
            e = edge;
        }
        Grid g;
        g.x0 = lo[0]; g.y0 = lo[1]; g.z0 = lo[2]; g.edge = e; g.inv_edge = 1.0 / e;
        g.nx = (int)nb[0]; g.ny = (int)nb[1]; g.nz = (int)nb[2];
        g.nbins = g.nx * g.ny * g.nz;
        g.max_half_l = maxh;
        *grid = g;
        // reset accumulators for the next rebuild
        for (int k = 0; k < 3; ++k) { acc[k] = 0xffffffffffffffffull; acc[3 + k] = 0ull; }
        acc[6] = 0ull;
        *counter = 0u;
    }
}

void launch_bbox(const Geom* geom, Ctrl* ctrl, Grid* grid, unsigned long long* acc,
                 unsigned int* counter, double edge, int cap_bins, int cap_cells, cudaStream_t st)
{
    int blocks = min(cdiv(cap_cells, 256), 592);
    k_bbox<<<max(blocks, 1), 256, 0, st>>>(geom, ctrl, grid, acc, counter, edge, cap_bins);
}

__device__ __forceinline__ int bin_coord(double x, double x0, double inv_edge, int nb)
{
    int b = (int)floor((x - x0) * inv_edge);
    return b < 0 ? 0 : (b >= nb ? nb - 1 : b);
}

__global__ void k_bin_count(const Geom* __restrict__ geom, const Ctrl* ctrl, const Grid* grid,
                            int* bin_count, int* key, int* slot)
{
    const int n = ctrl->n;
    const Grid g = *grid;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        Geom c = load_geom(geom, i);
        int bx = bin_coord(c.rx, g.x0, g.inv_edge, g.nx);
        int by = bin_coord(c.ry, g.y0, g.inv_edge, g.ny);
        int bz = bin_coord(c.rz, g.z0, g.inv_edge, g.nz);
        int k = (bz * g.ny + by) * g.nx + bx;
        if (k >= g.nbins) k = g.nbins - 1;
        key[i] = k;
        slot[i] = atomicAdd(&bin_count[k], 1);
    }
}

void launch_bin_count(const Geom* geom, const Ctrl* ctrl, const Grid* grid, int* bin_count,
                      int* key, int* slot, int cap_cells, cudaStream_t st)
{
    k_bin_count<<<max(cdiv(cap_cells, 256), 1), 256, 0, st>>>(geom, ctrl, grid, bin_count, key, slot);
}

__global__ void k_bin_scatter(const Geom* __restrict__ geom, const Ctrl* ctrl, const int* bin_start,
                              const int* key, const int* slot, int* sorted_cell, Geom* sorted_geom)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        int pos = bin_start[key[i]] + slot[i];
        sorted_cell[pos] = i;
        sorted_geom[pos] = load_geom(geom, i);
    }
}

void launch_bin_scatter(const Geom* geom, const Ctrl* ctrl, const int* bin_start, const int* key,
                        const int* slot, int* sorted_cell, Geom* sorted_geom, int cap_cells,
                        cudaStream_t st)
{
    k_bin_scatter<<<max(cdiv(cap_cells, 256), 1), 256, 0, st>>>(geom, ctrl, bin_start, key, slot,
                                                                 sorted_cell, sorted_geom);
}

// ---------------------------------------------------------------------------
// Exclusive scan (three passes: block sums, one-block scan of the sums,
// block scan + offset).  Up to 4096 * 4096 entries.
// ---------------------------------------------------------------------------
const int SCAN_T = 1024, SCAN_PER = 4, SCAN_TILE = SCAN_T * SCAN_PER;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sh_warp, int& total)
{
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh_warp[wid] = x;
    __syncthreads();
    if (wid == 0)
    {
        int w = (lane < (int)(blockDim.x >> 5)) ? sh_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        sh_warp[lane] = w;
    }
    __syncthreads();
    int warp_off = wid > 0 ? sh_warp[wid - 1] : 0;
    total = sh_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_off + x - v;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_sums(const int* __restrict__ in, const int* len_p,
                                                      int* block_sums)
{
    __shared__ int sh[32];
    const int len = *len_p;
    long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_PER;
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; ++k) if (base + k < len) s += in[base + k];
    int total;
    block_exclusive_scan(s, sh, total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_top(int* block_sums, int nblocks)
{
    __shared__ int sh[32];
    int base = threadIdx.x * SCAN_PER;
    int v[SCAN_PER], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; ++k) { v[k] = (base + k < nblocks) ? block_sums[base + k] : 0; s += v[k]; }
    int total;
    int off = block_exclusive_scan(s, sh, total);
#pragma unroll
    for (int k = 0; k < SCAN_PER; ++k) { if (base + k < nblocks) block_sums[base + k] = off; off += v[k]; }
    if (threadIdx.x == 0) block_sums[nblocks] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_final(const int* __restrict__ in, const int* len_p,
                                                       const int* block_sums, int* out, int nblocks)
{
    __shared__ int sh[32];
    const int len = *len_p;
    long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_PER;
    int v[SCAN_PER], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; ++k) { v[k] = (base + k < len) ? in[base + k] : 0; s += v[k]; }
    int total;
    int off = block_exclusive_scan(s, sh, total) + block_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_PER; ++k) { if (base + k < len) out[base + k] = off; off += v[k]; }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[len] = block_sums[nblocks];
}

// Arrays of at most SCAN_SINGLE_MAX entries: one block of SCAN_T threads, each
// summing a run of at most 64 consecutive entries, then writing its run's prefixes.
// One launch instead of three, for the many small scans of replicate batches.
const int SCAN_SINGLE_MAX = 1 << 16;

__global__ void __launch_bounds__(SCAN_T) k_scan_single(const int* __restrict__ in, const int* len_p, int* out)
{
    __shared__ int sh[32];
    const int len = *len_p;
    const int per = (len + SCAN_T - 1) / SCAN_T;
    const int b0 = min(threadIdx.x * per, len), b1 = min(b0 + per, len);
    int s = 0;
    for (int k = b0; k < b1; ++k) s += in[k];
    int total;
    int off = block_exclusive_scan(s, sh, total);
    for (int k = b0; k < b1; ++k) { const int v = in[k]; out[k] = off; off += v; }
    if (threadIdx.x == 0) out[len] = total;
}

size_t scan_block_sums_size(int cap) { return (size_t)cdiv(cap, SCAN_TILE) + 1; }

void launch_scan(const int* in, const int* len, int* out, int* block_sums, int cap, cudaStream_t st)
{
    if (cap <= SCAN_SINGLE_MAX)
    {
        k_scan_single<<<1, SCAN_T, 0, st>>>(in, len, out);
        return;
    }
    int nb = max(cdiv(cap, SCAN_TILE), 1);
    k_scan_sums<<<nb, SCAN_T, 0, st>>>(in, len, block_sums);
    k_scan_top<<<1, SCAN_T, 0, st>>>(block_sums, nb);
    k_scan_final<<<nb, SCAN_T, 0, st>>>(in, len, block_sums, out, nb);
}

// ---------------------------------------------------------------------------
// Pair build: one block per bin (grid-stride over bins), the bin's cells in
// groups of up to PB_G.  The block's threads sweep the flattened (own cell,
// candidate) products of the 27 surrounding bins with a cheap rejection test;
// the survivors go to a per-warp queue and are evaluated 32 at a time, so the
// exact FP64 distance runs on full warps instead of once per candidate for
// whichever lane needs it.  A survivor is kept when it passes the reference's
// two tests: centre distance < threshold + Ldiv + 2R and segment distance <
// threshold (mechanics.hpp:548-577).  The segment distance is always evaluated
// with the larger index as cell 1, as the reference's j < i loop does, so both
// cells of a pair reach the same decision.  Rows are filled in any order
// (shared-memory counters) and sorted by k_csr_fill.
//
// The rejection test is rigorous: every branch of dist_between_cells returns
// points r1 + s n1, r2 + t n2 with |s| <= h1, |t| <= h2, so the computed |d|
// is at least |r2 - r1| - h1 |n1| - h2 |n2| up to rounding (~1e-12 um at
// these coordinates).  A candidate is dropped only when, in FP32 with a
// 1e-4 um margin, |r2 - r1| > threshold + h1 max(1, |n1|^2) + h2 max(1, |n2|^2),
// i.e. when its |d| is certainly >= threshold.
// ---------------------------------------------------------------------------
const int PB_T = 128, PB_G = 128, PB_WARPS = PB_T / 32, PB_SLICE = 1 << 20;

struct PbShared {
    double rx[PB_G], ry[PB_G], rz[PB_G];
    float reach[PB_G];                  // h max(1, |n|^2)
    int cnt[PB_G];
    int q_own[PB_WARPS][64], q_pos[PB_WARPS][64];
};

__device__ __forceinline__ float pb_reach(double h, double nx, double ny, double nz)
{
    const float n2 = (float)(nx * nx + ny * ny + nz * nz);
    return (float)h * fmaxf(1.f, n2 * 1.000001f);
}

// exact tests for one queued (own, candidate) product
__device__ __forceinline__ void pb_exact(const Geom* __restrict__ sorted_geom, const int* __restrict__ sorted_cell,
                                         int base, int own, int pos, const BuildParams& bp, PbShared& sh,
                                         int* scratch)
{
    const Geom gm = sorted_geom[base + own], go = sorted_geom[pos];
    const int cm = sorted_cell[base + own], o = sorted_cell[pos];
    const Geom& gi = (cm > o) ? gm : go;
    const Geom& gj = (cm > o) ? go : gm;
    double cd = xnorm(xsub(x3(gi.rx, gi.ry, gi.rz), x3(gj.rx, gj.ry, gj.rz)));
    if (!(cd < bp.prefilter)) return;
    Dist d = dist_geom(gi, gj);
    if (xnorm(x3(d.dx, d.dy, d.dz)) < bp.threshold)
    {
        const int slot = atomicAdd(&sh.cnt[own], 1);
        if (slot < bp.cap_per_cell) scratch[(size_t)cm * bp.cap_per_cell + slot] = o;
    }
}

__global__ void __launch_bounds__(PB_T) k_pair_build(const Grid* grid, const int* __restrict__ bin_start,
                                                    const int* __restrict__ sorted_cell,
                                                    const Geom* __restrict__ sorted_geom, const Ctrl* ctrl,
                                                    BuildParams bp, int* scratch, int* count)
{
    __shared__ PbShared sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const Grid g = *grid;
    const int cap = bp.cap_per_cell;
    const float thr = (float)bp.threshold + 1e-4f;
    if (ctrl->status & ST_BIN_OVERFLOW)
    {
        // the cells do not fit a grid (k_bbox): an empty neighbor set, reported by the host
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ctrl->n; i += gridDim.x * blockDim.x) count[i] = 0;
        return;
    }
    for (int bin = blockIdx.x; bin < g.nbins; bin += gridDim.x)
    {
        const int s0 = bin_start[bin], s1 = bin_start[bin + 1];
        if (s0 == s1) continue;
        const int bx = bin % g.nx, by = (bin / g.nx) % g.ny, bz = bin / (g.nx * g.ny);
        for (int base = s0; base < s1; base += PB_G)
        {
            const int G = min(PB_G, s1 - base);
            __syncthreads();                                   // the previous group is done with sh
            for (int q = threadIdx.x; q < G; q += PB_T)
            {
                const Geom x = sorted_geom[base + q];
                sh.rx[q] = x.rx; sh.ry[q] = x.ry; sh.rz[q] = x.rz;
                sh.reach[q] = pb_reach(x.h, x.nx, x.ny, x.nz);
                sh.cnt[q] = 0;
            }
            __syncthreads();
            int qn = 0;                                        // this warp's queue length (warp-uniform)
            for (int dz = -1; dz <= 1; ++dz)
            {
                const int zz = bz + dz;
                if (zz < 0 || zz >= g.nz) continue;
                for (int dy = -1; dy <= 1; ++dy)
                {
                    const int yy = by + dy;
                    if (yy < 0 || yy >= g.ny) continue;
                    for (int dx = -1; dx <= 1; ++dx)
                    {
                        const int xx = bx + dx;
                        if (xx < 0 || xx >= g.nx) continue;
                        const int nbin = (zz * g.ny + yy) * g.nx + xx;
                        if (nbin >= g.nbins) continue;
                        const int nb0 = bin_start[nbin], nb1 = bin_start[nbin + 1];
                        // candidates in slices of PB_SLICE so G * len stays far from INT_MAX
                        for (int c0 = nb0; c0 < nb1; c0 += PB_SLICE)
                        {
                        const int total = G * min(PB_SLICE, nb1 - c0);
                        // warps take consecutive 32-product slices; every lane of a
                        // warp runs the same number of rounds.  Product idx is (own =
                        // idx % G, candidate = idx / G); both advance by PB_T per round,
                        // so they are stepped instead of divided.
                        int q = (warp * 32 + lane) / G, r = (warp * 32 + lane) % G;
                        const int dq = PB_T / G, dr = PB_T % G;
                        for (int w0 = warp * 32; w0 < total; w0 += PB_T)
                        {
                            const int idx = w0 + lane;
                            bool pass = false;
                            int own = 0, pos = 0;
                            const int own_r = r, cand_q = q;
                            r += dr; q += dq;
                            if (r >= G) { r -= G; q += 1; }
                            if (idx < total)
                            {
                                own = own_r;
                                pos = c0 + cand_q;
                                if (pos != base + own)
                                {
                                    const Geom& c = sorted_geom[pos];
                                    const double cx = __ldg(&c.rx), cy = __ldg(&c.ry), cz = __ldg(&c.rz);
                                    const float fx = (float)(cx - sh.rx[own]);
                                    const float fy = (float)(cy - sh.ry[own]);
                                    const float fz = (float)(cz - sh.rz[own]);
                                    const float L = thr + sh.reach[own]
                                                    + pb_reach(__ldg(&c.h), __ldg(&c.nx), __ldg(&c.ny), __ldg(&c.nz));
                                    pass = !(fx * fx + fy * fy + fz * fz > L * L);
                                }
                            }
                            const unsigned m = __ballot_sync(0xffffffffu, pass);
                            if (pass)
                            {
                                const int r = qn + __popc(m & lt);
                                sh.q_own[warp][r] = own;
                                sh.q_pos[warp][r] = pos;
                            }
                            qn += __popc(m);
                            if (qn >= 32)
                            {
                                qn -= 32;
                                __syncwarp();
                                const int eo = sh.q_own[warp][qn + lane], ep = sh.q_pos[warp][qn + lane];
                                __syncwarp();
                                pb_exact(sorted_geom, sorted_cell, base, eo, ep, bp, sh, scratch);
                            }
                        }
                        }
                    }
                }
            }
            __syncwarp();
            if (lane < qn) pb_exact(sorted_geom, sorted_cell, base, sh.q_own[warp][lane], sh.q_pos[warp][lane], bp, sh,
                                    scratch);
            __syncthreads();                                   // every count of the group is final
            for (int q = threadIdx.x; q < G; q += PB_T)
            {
                int cnt = sh.cnt[q];
                if (cnt > cap) { atomicOr((int*)&ctrl->status, (int)ST_NBR_OVERFLOW); cnt = cap; }
                count[sorted_cell[base + q]] = cnt;
            }
        }
    }
}

void launch_pair_build(const Grid* grid, const int* bin_start, const int* sorted_cell,
                       const Geom* sorted_geom, const Ctrl* ctrl, BuildParams bp, int* scratch,
                       int* count, int cap_bins, int num_sms, cudaStream_t st)
{
    int blocks = min(cap_bins, num_sms * 16);
    k_pair_build<<<max(blocks, 1), PB_T, 0, st>>>(grid, bin_start, sorted_cell, sorted_geom, ctrl, bp,
                                                  scratch, count);
}

// CSR rows: copy each cell's list and sort it ascending (deterministic order for
// the force reduction; the reference's table is i-major, j ascending).  One warp
// per row: an entry's rank is the number of smaller entries in the row (entries
// are distinct cell indices), counted with shuffles, and the entry lands at
// row_ptr[i] + rank.
const int CF_T = 256;

__global__ void __launch_bounds__(CF_T) k_csr_fill(const Ctrl* ctrl, const int* __restrict__ row_ptr,
                                                  const int* __restrict__ scratch, int cap, int* col, Ctrl* ctrl_w)
{
    const int n = ctrl->n;
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (CF_T / 32);
    for (int i = (blockIdx.x * CF_T + threadIdx.x) >> 5; i < n; i += nwarps)
    {
        const int r0 = row_ptr[i], len = row_ptr[i + 1] - r0;
        const int* src = scratch + (size_t)i * cap;
        for (int a = 0; a < len; a += 32)
        {
            const int v = (a + lane < len) ? src[a + lane] : INT_MAX;
            int rank = 0;
            for (int b = 0; b < len; b += 32)
            {
                const int w = (b + lane < len) ? src[b + lane] : INT_MAX;
#pragma unroll 8
                for (int q = 0; q < 32; ++q) rank += (__shfl_sync(0xffffffffu, w, q) < v) ? 1 : 0;
            }
            if (a + lane < len) col[r0 + rank] = v;
        }
        if (i == n - 1 && lane == 0) ctrl_w->n_dir = r0 + len;
    }
    if (n == 0 && blockIdx.x == 0 && threadIdx.x == 0) ctrl_w->n_dir = 0;
}

void launch_csr_fill(const Ctrl* ctrl, const int* row_ptr, const int* scratch, int cap, int* col, Ctrl* ctrl_w,
                     int cap_cells, cudaStream_t st)
{
    k_csr_fill<<<max(cdiv(cap_cells, CF_T / 32), 1), CF_T, 0, st>>>(ctrl, row_ptr, scratch, cap, col, ctrl_w);
}

// ---------------------------------------------------------------------------
// Pair force: G lanes per cell walk its CSR row; each lane evaluates the
// distance (larger index as cell 1) and the Hertz / JKR + hard-core magnitude
// of mechanics.hpp:1390-1659 (or :1209-1350 without adhesion), accumulates the
// cell's share of dE/dq, and the G partial sums are combined by xor shuffles.
// ---------------------------------------------------------------------------
// FP32 variant: segment distance (FP64 near-parallel branch kept), overlap,
// Hertz / JKR magnitude and direction in single precision
__device__ __forceinline__ PairOut pair_force_fp32(const Geom& gi, const Geom& gj, const ForceParams& fp,
                                                   const double* td, const double* tr)
{
    PairOut out;
    out.touch = false;
    Dist d = dist_geom_mixed(gi, gj);
    // the overlap from the FP64 distance vector, then the force law in FP32
    const double distd = sqrt((d.dx * d.dx + d.dy * d.dy) + d.dz * d.dz);
    const double overlap_d = 2 * fp.R - distd;
    if (!(overlap_d > 0)) return out;
    float dx = (float)d.dx, dy = (float)d.dy, dz = (float)d.dz;
    const float dist = (float)distd;
    const float R = (float)fp.R, max_overlap = (float)fp.max_overlap;
    float overlap = (float)overlap_d;
    float inv = 1.f / dist;
    float m;
    const double gamma = fp.adhesion ? fmin(gi.gamma, gj.gamma) : 0.0;
    if (fp.adhesion && gamma > 0)
    {
        // the JKR magnitude term1 - term2 cancels near the force balance, where most
        // adhering contacts sit: it keeps FP64 (table lookup included)
        m = (float)(fp.jkr_ng ? jkr_magnitude_variable(distd, gamma, fp, td) : jkr_magnitude(distd, gamma, fp, td, tr));
    }
    else if (overlap <= max_overlap) m = (float)fp.pf0 * overlap * sqrtf(overlap);
    else
    {
        m = (float)fp.pf2;
        if (!fp.adhesion) { float e = overlap - max_overlap; m += (float)fp.pf1 * e * sqrtf(e); }
    }
    if (fp.adhesion && overlap > max_overlap) { float e = overlap - max_overlap; m += (float)fp.pf1 * e * sqrtf(e); }
    out.vx = (double)(m * dx * inv); out.vy = (double)(m * dy * inv); out.vz = (double)(m * dz * inv);
    out.s = d.s; out.t = d.t; out.ovl = overlap; out.touch = true;
    return out;
}

// 2-D pair (2D/include/mechanics.hpp:448-547 and :572-670 with
// 2D/include/adhesion.hpp:403-448).  Returns p = cell i's translational dE/dq of the
// pair (Hertz v_ij minus strength * the JKR vector); i's torque share is s p and
// j's is (-p, -t p), projected per RK stage with the stage orientation.
__device__ __forceinline__ PairOut pair_force_2d(const Geom& gi, const Geom& gj, const ForceParams& fp,
                                                 bool adhere)
{
    PairOut out;
    out.touch = false;
    Dist d = dist_geom(gi, gj);
    const double mag = xnorm(x3(d.dx, d.dy, d.dz));
    const double overlap = 2 * fp.R - mag;
    if (!(overlap > 0)) return out;
    const double dirx = d.dx / mag, diry = d.dy / mag;
    double prefactor;
    if (overlap < fp.max_overlap) prefactor = fp.pf2d[0] * pow15(overlap);
    else prefactor = fp.pf2d[1] + fp.pf2d[2] * pow15(overlap - fp.max_overlap);
    double px = prefactor * dirx, py = prefactor * diry;
    if (adhere)
    {
        // overlap > 0 implies dist <= 2R
        const double term = M_PI * fp.R * (2 * fp.R - (mag <= fp.adh_mindist ? fp.adh_mindist : mag));
        px -= fp.adh_strength * (term * dirx);
        py -= fp.adh_strength * (term * diry);
    }
    out.vx = px; out.vy = py; out.vz = 0.0;
    out.s = d.s; out.t = d.t; out.ovl = overlap; out.touch = true;
    return out;
}

const int PF_T = 256, JKR_MAX = 512;

// Pass 1: G lanes per cell i walk the lower part of its sorted CSR row (j < i),
// evaluate each unordered pair once, keep i's share and write j's share
// (v, t) into the slot of i in row j (rev[k]).
template <int G, bool MIXED, int DIM>
__global__ void __launch_bounds__(PF_T) k_pair_force(const Geom* __restrict__ geom, const int* __restrict__ row_ptr,
                                                    const int* __restrict__ lower_end, const int* __restrict__ col,
                                                    const int* __restrict__ rev, Ctrl* ctrl, ForceParams fp,
                                                    const double* __restrict__ jkr_delta,
                                                    const double* __restrict__ jkr_radius, Gen6* fcc,
                                                    double4* __restrict__ jbuf)
{
    __shared__ double td[JKR_MAX], tr[JKR_MAX];
    if (ctrl->halted) return;
    for (int k = threadIdx.x; k < fp.jkr_n; k += blockDim.x) { td[k] = jkr_delta[k]; tr[k] = jkr_radius[k]; }
    __syncthreads();
    const int n = ctrl->n;
    const int lane = threadIdx.x & (G - 1);
    const unsigned gmask = (G == 32) ? 0xffffffffu
                                     : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
    const int groups_per_grid = gridDim.x * (blockDim.x / G);
    double ovl_max = 0.0;
    for (int cell = (blockIdx.x * blockDim.x + threadIdx.x) / G; cell < n; cell += groups_per_grid)
    {
        const Geom gc = load_geom(geom, cell);
        double acc[6] = {0, 0, 0, 0, 0, 0};
        const int r0 = row_ptr[cell], r1 = lower_end[cell];
        for (int k = r0 + lane; k < r1; k += G)
        {
            const int o = col[k];
            const Geom go = load_geom(geom, o);
            PairOut p;
            if (DIM == 2) p = pair_force_2d(gc, go, fp, fp.adhere[k] != 0);
            else p = MIXED ? pair_force_fp32(gc, go, fp, td, tr) : pair_force_fp64(gc, go, fp, td, tr);
            double4 js = make_double4(0.0, 0.0, 0.0, 0.0);
            if (p.touch)
            {
                acc[0] += p.vx; acc[1] += p.vy; acc[2] += p.vz;
                acc[3] += p.s * p.vx; acc[4] += p.s * p.vy; acc[5] += p.s * p.vz;
                js = make_double4(p.vx, p.vy, p.vz, p.t);
                ovl_max = fmax(ovl_max, p.ovl);
            }
            jbuf[rev[k]] = js;
        }
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
            for (int c = 0; c < 6; ++c) acc[c] += __shfl_xor_sync(gmask, acc[c], off, G);
        if (lane == 0)
        {
            Gen6 out;
            for (int c = 0; c < 6; ++c) out.f[c] = acc[c];
            fcc[cell] = out;
        }
    }
    if (fp.stats)
    {
        ovl_max = warp_max(ovl_max);
        if ((threadIdx.x & 31) == 0 && ovl_max > 0)
            atomicMax(&ctrl->st_ovl_bits[ctrl->iter & 1], (unsigned long long)__double_as_longlong(ovl_max));
    }
}

// Pass 2: each cell j adds the shares its higher-index neighbors left in the
// upper part of its row: (-v, -t v).
template <int G>
__global__ void __launch_bounds__(PF_T) k_pair_gather(const int* __restrict__ row_ptr, const int* __restrict__ lower_end,
                                                     const Ctrl* ctrl, const double4* __restrict__ jbuf, Gen6* fcc)
{
    const int n = ctrl->n;
    const int lane = threadIdx.x & (G - 1);
    const unsigned gmask = (G == 32) ? 0xffffffffu
                                     : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
    const int groups_per_grid = gridDim.x * (blockDim.x / G);
    for (int cell = (blockIdx.x * blockDim.x + threadIdx.x) / G; cell < n; cell += groups_per_grid)
    {
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int k = lower_end[cell] + lane; k < row_ptr[cell + 1]; k += G)
        {
            double4 js = jbuf[k];
            acc[0] -= js.x; acc[1] -= js.y; acc[2] -= js.z;
            acc[3] -= js.w * js.x; acc[4] -= js.w * js.y; acc[5] -= js.w * js.z;
        }
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
            for (int c = 0; c < 6; ++c) acc[c] += __shfl_xor_sync(gmask, acc[c], off, G);
        if (lane == 0)
        {
            Gen6 f = fcc[cell];
            for (int c = 0; c < 6; ++c) f.f[c] += acc[c];
            fcc[cell] = f;
        }
    }
}

void launch_pair_force(const Geom* geom, const int* row_ptr, const int* lower_end, const int* col, const int* rev,
                       Ctrl* ctrl, ForceParams fp, const double* jkr_delta, const double* jkr_radius,
                       Gen6* fcc, double4* jbuf, int lanes, int mixed, int cap_cells, cudaStream_t st,
                       int with_gather, int dims)
{
    int blocks = max(cdiv((long long)cap_cells * lanes, PF_T), 1);
#define PF_CASE(G) \
    if (lanes == G) { \
        if (dims == 2) k_pair_force<G, false, 2><<<blocks, PF_T, 0, st>>>(geom, row_ptr, lower_end, col, rev, ctrl, fp, jkr_delta, jkr_radius, fcc, jbuf); \
        else if (mixed) k_pair_force<G, true, 3><<<blocks, PF_T, 0, st>>>(geom, row_ptr, lower_end, col, rev, ctrl, fp, jkr_delta, jkr_radius, fcc, jbuf); \
        else k_pair_force<G, false, 3><<<blocks, PF_T, 0, st>>>(geom, row_ptr, lower_end, col, rev, ctrl, fp, jkr_delta, jkr_radius, fcc, jbuf); \
        if (with_gather) k_pair_gather<G><<<blocks, PF_T, 0, st>>>(row_ptr, lower_end, ctrl, jbuf, fcc); \
        return; }
    PF_CASE(4) PF_CASE(8) PF_CASE(16) PF_CASE(32)
#undef PF_CASE
}

// Reverse slots and the end of the lower part of each sorted CSR row: for an
// entry (i, j) with j < i, rev = position of i in row j.
// Reverse indices and the lower part of each row, one warp per row: lower_end[i]
// is the first entry with j >= i (rows are sorted), and every lower entry (i, j)
// finds the position of i in row j by binary search.
__global__ void __launch_bounds__(CF_T) k_csr_rev(const Ctrl* ctrl, const int* __restrict__ row_ptr,
                                                 const int* __restrict__ col, int* lower_end, int* rev)
{
    const int n = ctrl->n;
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (CF_T / 32);
    for (int i = (blockIdx.x * CF_T + threadIdx.x) >> 5; i < n; i += nwarps)
    {
        const int r0 = row_ptr[i], r1 = row_ptr[i + 1];
        int lower = 0;
        for (int k0 = r0; k0 < r1; k0 += 32)
        {
            const int k = k0 + lane;
            const int j = k < r1 ? col[k] : INT_MAX;
            const bool lo = j < i;
            lower += __popc(__ballot_sync(0xffffffffu, lo));
            if (lo)
            {
                int a = row_ptr[j], b = row_ptr[j + 1];
                while (a < b) { const int mid = (a + b) >> 1; if (col[mid] < i) a = mid + 1; else b = mid; }
                rev[k] = a;
            }
        }
        if (lane == 0) lower_end[i] = r0 + lower;
    }
}

void launch_csr_rev(const Ctrl* ctrl, const int* row_ptr, const int* col, int* lower_end, int* rev,
                    int cap_cells, cudaStream_t st)
{
    k_csr_rev<<<max(cdiv(cap_cells, CF_T / 32), 1), CF_T, 0, st>>>(ctrl, row_ptr, col, lower_end, rev);
}

// ---------------------------------------------------------------------------
// Screened pair pass over the pair records (one per unordered pair: cell i, its
// partner j < i, the lower CSR entry k and the partner's entry rev[k]; the larger
// index is cell 1, as in the reference's j < i loop).  The screen is a lower
// bound on the centreline distance: for any unit vector a, the gap between the
// projections of the two segments on a,
//     a . (c_j - c_i) - h_i |a . n_i| - h_j |a . n_j|,
// bounds their distance from below.  a is the closest-point direction of a
// single-precision estimate, so the bound is nearly tight, and it is evaluated
// in FP64, so it is rigorous (may_touch).  The exact pair force writes the pair's
// two shares: (v, s) into the lower entry and (v, t) into the partner's entry.
// The first attempt sums a cell's whole row in CSR order.
// ---------------------------------------------------------------------------
const int PS_T = 256, PS_TILE_MAX = 2048;

template <bool MIXED>
__device__ __forceinline__ void zero_shares(double4* jbuf, int k, int r)
{
    if (MIXED)
    {
        float4* fb = reinterpret_cast<float4*>(jbuf);
        fb[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        fb[r] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    else
    {
        jbuf[k] = make_double4(0.0, 0.0, 0.0, 0.0);
        jbuf[r] = make_double4(0.0, 0.0, 0.0, 0.0);
    }
}

// One pass per iteration over the pair records.  A refresh iteration (the active
// list is stale: after a rebuild, an upload or a division, or once the cells may
// have moved by half the skin since the last refresh, 2 * drift >= skin) screens
// every pair with the rigorous bound of may_touch, zeroes the shares of the pairs
// beyond 2R + skin, computes the others and lists them as the new active pairs;
// the other iterations compute the active pairs only.  A pair left out stays
// beyond 2R until the next refresh (its distance can fall by at most
// 2 * drift < skin), so its force is exactly zero in every force law of the
// reference (all need overlap > 0).  Every share slot is written by exactly one
// pair, so the order of the active list changes no result.  The last block
// installs a new list and clears the drift.
// the friction part of a touching pair's shares (FP64): v -= the force on i under the
// decision at the attempt's positions; a candidate also records the change of v when the
// decision flips, and is listed for the stage checks
__device__ __forceinline__ void friction_shares(const Geom& gi, const Geom& gj, const int4& pr, const ForceParams& fp,
                                                const Dist& d, double dist, double4& own, double4& other)
{
    const int i = pr.x, j = pr.y;
    const X3 dv = x3(d.dx, d.dy, d.dz);
    const Vel ui = fp.vel[i], uj = fp.vel[j];
    const double eta = fmin(fp.feta[i], fp.feta[j]);
    double rv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) rv[c] = (ui.v[c] + d.s * ui.v[3 + c]) - (uj.v[c] + d.t * uj.v[3 + c]);
    const bool cand = fp.surface && fabs(__ddiv_rn(d.dz, dist)) < 1e-3;
    bool flat0 = false;
    if (cand)
    {
        const double lim = 1.01 * fp.R;
        flat0 = __dadd_rn(gi.rz, __dmul_rn(d.s, gi.nz)) < lim && __dadd_rn(gj.rz, __dmul_rn(d.t, gj.nz)) < lim;
    }
    double f[3];
    friction_force(dv, dist, flat0, rv, eta, fp, f);
    own.x -= f[0]; own.y -= f[1]; own.z -= f[2];
    other.x -= f[0]; other.y -= f[1]; other.z -= f[2];
    if (cand)
    {
        double g[3];
        friction_force(dv, dist, !flat0, rv, eta, fp, g);
        const double4 delta = make_double4(-(g[0] - f[0]), -(g[1] - f[1]), -(g[2] - f[2]), 0.0);
        fp.fbuf[pr.z] = delta;
        fp.fbuf[pr.w] = delta;
        const int m = FR_CAND | (flat0 ? FR_D0 : 0);
        fp.fmask[pr.z] = m;
        fp.fmask[pr.w] = m;
    }
    else
    {
        fp.fmask[pr.z] = 0;
        fp.fmask[pr.w] = 0;
    }
}

template <bool MIXED, int DIM>
__device__ __forceinline__ void pair_shares(const Geom& gi, const Geom& gj, const int4& pr, const ForceParams& fp,
                                            const double* __restrict__ td, const double* __restrict__ tr,
                                            double4* __restrict__ jbuf, double& ovl_max, bool* fr_cand = nullptr)
{
    const int k = pr.z, r = pr.w;
    PairOut p;
    if (DIM == 2) p = pair_force_2d(gi, gj, fp, fp.adhere[k] != 0);
    else p = MIXED ? pair_force_fp32(gi, gj, fp, td, tr) : pair_force_fp64(gi, gj, fp, td, tr);
    if (MIXED)
    {
        // mixed precision: the shares are single-precision forces, stored as such
        float4* fb = reinterpret_cast<float4*>(jbuf);
        float4 own = make_float4(0.f, 0.f, 0.f, 0.f), other = own;
        if (p.touch)
        {
            own = make_float4((float)p.vx, (float)p.vy, (float)p.vz, (float)p.s);
            other = make_float4((float)p.vx, (float)p.vy, (float)p.vz, (float)p.t);
            ovl_max = fmax(ovl_max, p.ovl);
        }
        fb[k] = own;
        fb[r] = other;
    }
    else
    {
        double4 own = make_double4(0.0, 0.0, 0.0, 0.0), other = own;
        if (p.touch)
        {
            own = make_double4(p.vx, p.vy, p.vz, p.s);
            other = make_double4(p.vx, p.vy, p.vz, p.t);
            ovl_max = fmax(ovl_max, p.ovl);
            if (DIM == 3 && fp.fric)
            {
                const Dist d = {p.dx, p.dy, p.dz, p.s, p.t};
                friction_shares(gi, gj, pr, fp, d, p.dist, own, other);
                if (fr_cand) *fr_cand = (fp.fmask[k] & FR_CAND) != 0;
            }
        }
        else if (DIM == 3 && fp.fric)
        {
            fp.fmask[k] = 0;
            fp.fmask[r] = 0;
        }
        jbuf[k] = own;
        jbuf[r] = other;
    }
}

// With PROPOSE the pass also makes the iteration's step-size proposal
// (mlp_propose_block). Its features read the previous iteration's overlap maximum
// (st_ovl_bits of the other parity, which no block of this pass writes), so the
// proposal depends on nothing this pass computes: the grid's last block makes it
// while the other blocks stride over the pairs, and its chain of dependent reads
// and three network layers runs beside the pair work instead of after it. A grid of
// one block computes its pairs first and proposes at the end. The proposal is a
// template parameter so that the passes without it carry none of its code, and the
// bound of two resident blocks per SM (at most 128 registers) holds the pair loop's
// occupancy whatever the proposal adds.
template <bool MIXED, int DIM, bool PROPOSE>
__global__ void __launch_bounds__(PS_T, 2) k_pair_pass(const Geom* __restrict__ geom, const int4* __restrict__ pairs,
                                                      Ctrl* ctrl, ForceParams fp, const double* __restrict__ td,
                                                      const double* __restrict__ tr, double4* __restrict__ jbuf,
                                                      int* __restrict__ surv, StepParams sp,
                                                      const float* __restrict__ mlp_w)
{
    __shared__ bool last;
    if (ctrl->halted) return;
    const bool split = PROPOSE && gridDim.x > 1;
    const bool proposer = split && blockIdx.x == gridDim.x - 1;
    const int work_blocks = split ? gridDim.x - 1 : gridDim.x;
    const bool refresh = !ctrl->screen_valid || !(2.0 * ctrl->drift * (1.0 + 1e-6) + 1e-9 < fp.skin);
    const int lane = threadIdx.x & 31;
    const int stride = work_blocks * blockDim.x;
    double ovl_max = 0.0;
    if (proposer)
        mlp_propose_block(ctrl, sp, mlp_w);
    else if (refresh)
    {
        const int n_pairs = ctrl->n_dir >> 1;
        const double limit = 2 * fp.R + fp.skin;
        // warp-uniform rounds, so that every ballot covers all 32 lanes
        for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n_pairs; base += stride)
        {
            const int p = base + lane;
            bool keep = false;
            int4 pr = make_int4(0, 0, 0, 0);
            Geom gi, gj;
            if (p < n_pairs)
            {
                pr = pairs[p];                      // (i, j, lower entry k, partner entry)
                gi = load_geom(geom, pr.x);
                gj = load_geom(geom, pr.y);
                keep = may_touch(gi, gj, limit);
                if (!keep)
                {
                    zero_shares<MIXED>(jbuf, pr.z, pr.w);
                    if (!MIXED && DIM == 3 && fp.fric) { fp.fmask[pr.z] = 0; fp.fmask[pr.w] = 0; }
                }
            }
            // warp-aggregated append of the active pairs
            const unsigned mask = __ballot_sync(0xffffffffu, keep);
            int pos = 0;
            if (lane == 0 && mask) pos = atomicAdd(&ctrl->n_surv_next, __popc(mask));
            pos = __shfl_sync(0xffffffffu, pos, 0);
            if (keep)
            {
                surv[pos + __popc(mask & ((1u << lane) - 1u))] = p;
                bool cand = false;
                pair_shares<MIXED, DIM>(gi, gj, pr, fp, td, tr, jbuf, ovl_max, &cand);
                if (cand) fp.fr_list[atomicAdd(&ctrl->fr_ncand_next, 1)] = p;
            }
        }
    }
    else
    {
        const int m = ctrl->n_surv;
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += stride)
        {
            const int p = surv[q];
            const int4 pr = pairs[p];
            bool cand = false;
            pair_shares<MIXED, DIM>(load_geom(geom, pr.x), load_geom(geom, pr.y), pr, fp, td, tr, jbuf, ovl_max, &cand);
            if (cand) fp.fr_list[atomicAdd(&ctrl->fr_ncand_next, 1)] = p;
        }
    }
    if (fp.stats && !proposer)
    {
        ovl_max = warp_max(ovl_max);
        if (lane == 0 && ovl_max > 0)
            atomicMax(&ctrl->st_ovl_bits[ctrl->iter & 1], (unsigned long long)__double_as_longlong(ovl_max));
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        last = atomicAdd(&ctrl->surv_blocks, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    if (threadIdx.x == 0)
    {
        __threadfence();
        if (refresh)
        {
            ctrl->n_surv = atomicAdd(&ctrl->n_surv_next, 0);
            ctrl->n_surv_next = 0;
            ctrl->screen_valid = 1;
            ctrl->drift = 0.0;
        }
        if (fp.fric)
        {
            // the candidates of this pass; no stage has a changed decision yet
            ctrl->fr_ncand = atomicAdd(&ctrl->fr_ncand_next, 0);
            ctrl->fr_ncand_next = 0;
            ctrl->fr_nflip = 0;
        }
        ctrl->surv_blocks = 0u;
    }
    if (PROPOSE && !split)
    {
        __syncthreads();
        mlp_propose_block(ctrl, sp, mlp_w);
    }
}

// The pair list visits cells in `order` (the cell list's bin order after a rebuild,
// else index order): pairs of one region of space are screened together, so each
// cell's record is fetched once and reused from the caches by its neighbours' pairs.

__global__ void k_lower_counts(const Ctrl* ctrl, const int* __restrict__ row_ptr, const int* __restrict__ lower_end,
                               const int* __restrict__ order, int* count)
{
    const int n = ctrl->n;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    {
        const int i = order ? order[q] : q;
        count[q] = lower_end[i] - row_ptr[i];
    }
}

// a new pair list makes the active list stale (block 0 marks it)
__global__ void k_pair_list_fill(Ctrl* ctrl, const int* __restrict__ row_ptr, const int* __restrict__ lower_end,
                                 const int* __restrict__ col, const int* __restrict__ rev,
                                 const int* __restrict__ order, const int* __restrict__ start, int4* pairs)
{
    const int n = ctrl->n;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->screen_valid = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    {
        const int i = order ? order[q] : q;
        const int r0 = row_ptr[i], p0 = start[q];
        for (int k = r0; k < lower_end[i]; ++k) pairs[p0 + (k - r0)] = make_int4(i, col[k], k, rev[k]);
    }
}

void launch_pair_list(const Ctrl* ctrl, const int* row_ptr, const int* lower_end, const int* col, const int* rev,
                      int* count, int* start, int* block_sums, int4* pairs, int cap_cells, cudaStream_t st,
                      const int* order)
{
    const int blocks = max(cdiv(cap_cells, 256), 1);
    k_lower_counts<<<blocks, 256, 0, st>>>(ctrl, row_ptr, lower_end, order, count);
    launch_scan(count, &ctrl->n, start, block_sums, cap_cells, st);
    k_pair_list_fill<<<blocks, 256, 0, st>>>(const_cast<Ctrl*>(ctrl), row_ptr, lower_end, col, rev, order, start,
                                             pairs);
}

// total dE/dq of each cell from the two shares of every pair (the API paths;
// the loop's first attempt does the same sum itself)
__global__ void k_pair_sum_rows(const int* __restrict__ row_ptr, const int* __restrict__ lower_end, const Ctrl* ctrl,
                                const double4* __restrict__ jbuf, Gen6* fcc, int f32);

void launch_pair_screened(const Geom* geom, const int* row_ptr, const int* lower_end, const int* col,
                          const int* rev, Ctrl* ctrl, ForceParams fp, const double* jkr_delta,
                          const double* jkr_radius, Gen6* fcc, double4* jbuf, int mixed, int max_entries,
                          int cap_cells, int num_sms, cudaStream_t st, int with_sum, int dims, int tile,
                          int blocks_per_sm, const int4* pairs, int* surv, const StepParams* sp,
                          const float* mlp_w)
{
    // sp (the loop's pass): the last block also runs the step-size proposal
    StepParams spv{};
    if (sp) spv = *sp;
    const int propose = (sp && sp->stats_on) ? 1 : 0;
    // grid: at least `tile` pairs per block, at most the blocks that are resident at
    // once (blocks_per_sm caps them per SM); the blocks stride over the pairs
    tile = tile <= 0 ? 1024 : min(tile, PS_TILE_MAX);
    const int max_pairs = max(max_entries / 2, 1);
    const bool f32 = mixed && dims != 2;
    auto grid = [&](const void* fn, int& occ_cache) {
        if (occ_cache == 0)
        {
            int occ = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, PS_T, 0);
            occ_cache = max(occ, 1);
        }
        const int per_sm = blocks_per_sm > 0 ? min(blocks_per_sm, occ_cache) : occ_cache;
        return max(1, min(cdiv(max_pairs, tile), num_sms * per_sm));
    };
    // resident blocks per SM of each instantiation (without, with the proposal)
    static int occ2[2] = {0, 0}, occ3m[2] = {0, 0}, occ3[2] = {0, 0};
#define PX_ARGS geom, pairs, ctrl, fp, jkr_delta, jkr_radius, jbuf, surv, spv, mlp_w
#define PX_LAUNCH(M, D, P, occ) \
    k_pair_pass<M, D, P><<<grid((const void*)k_pair_pass<M, D, P>, occ[P ? 1 : 0]), PS_T, 0, st>>>(PX_ARGS)
    if (dims == 2)
    {
        if (propose) PX_LAUNCH(false, 2, true, occ2);
        else PX_LAUNCH(false, 2, false, occ2);
    }
    else if (f32)
    {
        if (propose) PX_LAUNCH(true, 3, true, occ3m);
        else PX_LAUNCH(true, 3, false, occ3m);
    }
    else
    {
        if (propose) PX_LAUNCH(false, 3, true, occ3);
        else PX_LAUNCH(false, 3, false, occ3);
    }
#undef PX_LAUNCH
#undef PX_ARGS
    if (with_sum)
        k_pair_sum_rows<<<max(cdiv(cap_cells, 128), 1), 128, 0, st>>>(row_ptr, lower_end, ctrl, jbuf, fcc, f32);
}

// to_adhere (2D/include/simulation.hpp:242-258, one group in the adhesion map):
// for each lower entry (i, j < i), dist of the (i, j) row > R + Rcell and < 2R
__global__ void k_adhere_flags(const Ctrl* ctrl, const int* __restrict__ row_ptr, const int* __restrict__ col,
                               const Geom* __restrict__ geom, double R, double Rcell, unsigned char* adhere)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const Geom gi = load_geom(geom, i);
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
        {
            const int j = col[k];
            unsigned char a = 0;
            if (j < i)
            {
                Dist d = dist_geom(gi, load_geom(geom, j));
                const double dist = xnorm(x3(d.dx, d.dy, d.dz));
                a = (dist > R + Rcell && dist < 2 * R) ? 1 : 0;
            }
            adhere[k] = a;
        }
    }
}

void launch_adhere_flags(const Ctrl* ctrl, const int* row_ptr, const int* col, const Geom* geom, double R,
                         double Rcell, unsigned char* adhere, int cap_cells, cudaStream_t st)
{
    k_adhere_flags<<<max(cdiv(cap_cells, 128), 1), 128, 0, st>>>(ctrl, row_ptr, col, geom, R, Rcell, adhere);
}

// the reference's 2-D dE/dq (cellCellRepulsiveForces + cellCellAdhesiveForces) from the
// pair sums F = sum p and S = sum s p: torque S - (n . S) n at the current orientation
__global__ void k_pair_dEdq_2d(const Geom* __restrict__ geom, const Gen6* __restrict__ fcc, const Ctrl* ctrl,
                               double* cm)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const Geom g = load_geom(geom, i);
        const Gen6 f = fcc[i];
        const double w = g.nx * f.f[3] + g.ny * f.f[4];
        cm[i] = f.f[0];
        cm[(size_t)n + i] = f.f[1];
        cm[(size_t)2 * n + i] = f.f[3] - w * g.nx;
        cm[(size_t)3 * n + i] = f.f[4] - w * g.ny;
    }
}

void launch_pair_dEdq_2d(const Geom* geom, const Gen6* fcc, const Ctrl* ctrl, double* cm, int cap_cells,
                         cudaStream_t st)
{
    k_pair_dEdq_2d<<<max(cdiv(cap_cells, 256), 1), 256, 0, st>>>(geom, fcc, ctrl, cm);
}

// ---------------------------------------------------------------------------
// RK attempt: one thread per cell runs every stage of stepRungeKuttaAdaptive
// (mechanics.hpp:2406-2612) in registers.  3-D pair forces are stage-invariant
// (the table is not refreshed between stages and include_constraint = false,
// mechanics.hpp:2064), so each stage needs only the cell's own state, its
// precomputed pair force and the surface terms.
// ---------------------------------------------------------------------------
const int AT_T = 128;

__device__ __forceinline__ void normalize_n(double y[6])
{
    double nrm = sqrt((y[3] * y[3] + y[4] * y[4]) + y[5] * y[5]);
    y[3] /= nrm; y[4] /= nrm; y[5] /= nrm;
    if (y[5] < 0) { y[3] = -y[3]; y[4] = -y[4]; y[5] = -y[5]; }
}

// getVelocities (mechanics.hpp:2011-2347) of one cell at state y; f0 = -dE/dq of
// the (stage-invariant) pair forces plus noise
__device__ __forceinline__ void cell_velocity(const StepParams& sp, bool a2, const double y[6],
                                              double l, double h, double eta0, double eta1, double sigma0,
                                              const Vel* __restrict__ drp, const double f0[6], double v[6])
{
    const MechParams& P = sp.mp;
    double ss = a2 ? __longlong_as_double(0x7ff8000000000000ll) : (P.R - y[2]) / y[5];
    EndPow w;
    w.p = w.q = w.sp = w.sq = 0.0;
    if (!a2) w = end_pows(y[2], y[5], P.R, h, ss);
    double rep2 = 0, rep5 = 0, adh2 = 0, adh5 = 0;
    if (!P.no_surface) surface_dEdq(P, a2, y[2], y[5], l, h, sigma0, ss, w, rep2, rep5, adh2, adh5);
    double f[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) f[c] = f0[c];
    f[2] = (f[2] - rep2) - adh2;
    f[5] = (f[5] - rep5) - adh5;
    velocity_solve(P, a2, y, l, h, eta0, eta1, ss, w, drp, f, v);
}

// Mixed precision: a cell in surface contact (and not lying on the substrate) takes the
// FP32 contact branch (velocity_contact_f32); the others keep the FP64 branches (i) and
// (ii), whose surface forces are zero off the surface and the horizontal shortcut on it
__device__ __forceinline__ void cell_velocity_f32(const StepParams& sp, bool a2, const double y[6],
                                                  double l, double h, double eta0, double eta1, double sigma0,
                                                  const Vel* __restrict__ drp, const double f0[6], double v[6])
{
    const MechParams& P = sp.mp;
    const bool contacting = surface_contact(P, a2, y, h);
    if (!P.no_surface && contacting && !a2)
    {
        velocity_contact_f32(P, y, l, h, eta0, eta1, sigma0, drp, f0, v);
        return;
    }
    double f[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) f[c] = f0[c];
    if (!P.no_surface && a2)
    {
        double rep2 = 0, adh2 = 0;
        surface_dEdq_flat(P, y[2], l, sigma0, rep2, adh2);
        f[2] = (f[2] - rep2) - adh2;
    }
    velocity_free_or_flat(P, contacting, y, l, eta0, eta1, drp, f, v);
}

template <bool F32>
__device__ __forceinline__ void cell_velocity_p(const StepParams& sp, bool a2, const double y[6], double l,
                                                double h, double eta0, double eta1, double sigma0,
                                                const Vel* __restrict__ drp, const double f0[6], double v[6])
{
    if constexpr (F32) cell_velocity_f32(sp, a2, y, l, h, eta0, eta1, sigma0, drp, f0, v);
    else cell_velocity(sp, a2, y, l, h, eta0, eta1, sigma0, drp, f0, v);
}

// -dE/dq of the pair forces (getConservativeForces, mechanics.hpp:1768) plus the
// attempt's noise (mechanics.hpp:2489-2510, forces += noise at :2066)
template <bool NOISE>
__device__ __forceinline__ void base_force(const StepParams& sp, const Gen6& cc, int iter, int attempt, int i,
                                           double f0[6])
{
#pragma unroll
    for (int c = 0; c < 6; ++c) f0[c] = -cc.f[c];
    if (NOISE)
    {
        for (int k = 0; k < 3; ++k)
        {
            uint32_t x[4] = {(uint32_t)iter, (uint32_t)attempt, (uint32_t)i, (uint32_t)k};
            philox4x32_10(x, (uint32_t)sp.seed, (uint32_t)(sp.seed >> 32) ^ RNG_PURPOSE_NOISE);
            double u0 = philox_u01(x[0], x[1]), u1 = philox_u01(x[2], x[3]);
            f0[2 * k] += -sp.noise_max[2 * k] + 2 * sp.noise_max[2 * k] * u0;
            f0[2 * k + 1] += -sp.noise_max[2 * k + 1] + 2 * sp.noise_max[2 * k + 1] * u1;
        }
    }
}

// 2-D noise of one attempt (2D/include/mechanics.hpp:1760-1771): uniform on
// [-max, max] for (rx, ry, nx, ny), from the 3-D counter slots 0, 1, 3, 4
__device__ __forceinline__ void noise_2d(const StepParams& sp, int iter, int attempt, int i, double nz[4])
{
    double u[6];
    for (int k = 0; k < 3; ++k)
    {
        uint32_t x[4] = {(uint32_t)iter, (uint32_t)attempt, (uint32_t)i, (uint32_t)k};
        philox4x32_10(x, (uint32_t)sp.seed, (uint32_t)(sp.seed >> 32) ^ RNG_PURPOSE_NOISE);
        u[2 * k] = philox_u01(x[0], x[1]);
        u[2 * k + 1] = philox_u01(x[2], x[3]);
    }
    const double m = sp.max_noise_2d;
    nz[0] = -m + 2 * m * u[0]; nz[1] = -m + 2 * m * u[1];
    nz[2] = -m + 2 * m * u[3]; nz[3] = -m + 2 * m * u[4];
}

// 2-D getVelocities (2D/include/mechanics.hpp:1503-1667) at stage orientation (y3, y4):
// dE/dq = (F, S - (n . S) n) + noise from the pair sums cc = (F, S); v = -dE/dq / (K, L)
// with K = l (eta0 + eta1 rho_c / R), L = l^3 (...) / 12 (:264-279)
__device__ __forceinline__ void velocity_2d(const StepParams& sp, const double y[6], double l, double eta0,
                                            double eta1, const Gen6& cc, const double nz[4], double v[6])
{
    const double drag = eta0 + eta1 * sp.rho_c / sp.mp.R;
    const double K = l * drag, L = l * l * l * drag / 12;
    const double w = y[3] * cc.f[3] + y[4] * cc.f[4];
    const double d0 = cc.f[0] + nz[0], d1 = cc.f[1] + nz[1];
    const double d2 = (cc.f[3] - w * y[3]) + nz[2], d3 = (cc.f[4] - w * y[4]) + nz[3];
    v[0] = -d0 / K; v[1] = -d1 / K; v[2] = 0.0;
    v[3] = -d2 / L; v[4] = -d3 / L; v[5] = 0.0;
}

__device__ __forceinline__ Gen6 load_gen6(const Gen6* __restrict__ g, int i)
{
    const double2* p = reinterpret_cast<const double2*>(g + i);
    double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    Gen6 o;
    o.f[0] = a.x; o.f[1] = a.y; o.f[2] = b.x; o.f[3] = b.y; o.f[4] = c.x; o.f[5] = c.y;
    return o;
}

// dE/dq of cell i: the share of its lower neighbors (written by k_pair_force) plus
// the shares its higher-index neighbors left in the upper part of its row
__device__ __forceinline__ Gen6 gather_pair_force(const Gen6* fcc, const int* __restrict__ row_ptr,
                                                  const int* __restrict__ lower_end,
                                                  const double4* __restrict__ jbuf, int i)
{
    Gen6 f = fcc[i];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int k = lower_end[i]; k < row_ptr[i + 1]; ++k)
    {
        double4 js = jbuf[k];
        acc[0] -= js.x; acc[1] -= js.y; acc[2] -= js.z;
        acc[3] -= js.w * js.x; acc[4] -= js.w * js.y; acc[5] -= js.w * js.z;
    }
    for (int c = 0; c < 6; ++c) f.f[c] += acc[c];
    return f;
}

__device__ __forceinline__ double4 widen(const double4& v) { return v; }
__device__ __forceinline__ double4 widen(const float4& v)
{
    return make_double4((double)v.x, (double)v.y, (double)v.z, (double)v.w);
}

// dE/dq of cell i from both shares of every pair in its row: (v, s v) from its lower
// entries, (-v, -t v) from the partners' entries, in CSR order.  Shares are stored
// as double4, or as float4 (mixed precision), summed in FP64 either way.
template <class SHARE>
__device__ __forceinline__ Gen6 sum_row_shares(const int* __restrict__ row_ptr, const int* __restrict__ lower_end,
                                               const SHARE* __restrict__ jbuf, int i)
{
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int le = lower_end[i], r1 = row_ptr[i + 1];
    for (int k = row_ptr[i]; k < le; ++k)
    {
        const double4 js = widen(jbuf[k]);
        acc[0] += js.x; acc[1] += js.y; acc[2] += js.z;
        acc[3] += js.w * js.x; acc[4] += js.w * js.y; acc[5] += js.w * js.z;
    }
    for (int k = le; k < r1; ++k)
    {
        const double4 js = widen(jbuf[k]);
        acc[0] -= js.x; acc[1] -= js.y; acc[2] -= js.z;
        acc[3] -= js.w * js.x; acc[4] -= js.w * js.y; acc[5] -= js.w * js.z;
    }
    Gen6 f;
    for (int c = 0; c < 6; ++c) f.f[c] = acc[c];
    return f;
}

__global__ void k_pair_sum_rows(const int* __restrict__ row_ptr, const int* __restrict__ lower_end, const Ctrl* ctrl,
                                const double4* __restrict__ jbuf, Gen6* fcc, int f32)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        fcc[i] = f32 ? sum_row_shares(row_ptr, lower_end, reinterpret_cast<const float4*>(jbuf), i)
                     : sum_row_shares(row_ptr, lower_end, jbuf, i);
}

// Step-size controller, run once per attempt by the last block
// (simulation.hpp:1690-1769; the final re-run is accepted unconditionally).
// commit: the final step copies an accepted proposal (no RK evaluation of its own)
__device__ void controller_finish(Ctrl* c, const StepParams& sp, int kind, double E, bool commit = false)
{
    if (!commit) c->attempts += 1;
    if (kind == MODE_TRIAL)
    {
        c->last_trial_error = E;
        bool exceeded = E > 1.0;
        c->first_passed = !exceeded;
        if (exceeded) c->rejected += 1;
        if (sp.log_cap > 0)
        {
            // complete the feature row of this iteration: the log ratio of the largest
            // dt the error model accepts, and of this attempt's dt, to the last accepted dt
            float* row = sp.log_buf + (size_t)(c->log_rows % sp.log_cap) * MLP_LOG_COLS;
            row[32] = (float)(-sp.inv_q1 * log(E));
            row[33] = (float)log(c->dt / c->dt_prev);
            row[34] = (float)log10(E);
            row[35] = exceeded ? 0.f : 1.f;
            c->log_rows += 1;
        }
        if (sp.propose && !exceeded)
        {
            // the proposal passed the error test: accept its candidate state as is
            c->mode = MODE_COMMIT;
            c->tries = 0;
            c->attempt = 1;
            return;
        }
        double factor = 0.9 * pow(1.0 / E, sp.inv_q1);
        if (factor >= 10) factor = 10;
        else if (factor < 0.2) factor = 0.2;
        c->factor = factor;
        c->tries = 0;
        c->attempt = 1;
        if (exceeded && 0 < sp.max_tries) { c->mode = MODE_RETRY; c->dt_try = c->dt * factor; return; }
    }
    else if (kind == MODE_RETRY)
    {
        c->retries += 1;
        c->attempt += 1;
        bool exceeded = E > 1.0;
        double factor = c->factor * (0.9 * pow(1.0 / E, sp.inv_q1));
        bool brk = false;
        if (factor >= 10) { factor = 10; brk = true; }
        else if (factor < 0.2) { factor = 0.2; brk = true; }
        c->factor = factor;
        if (!brk)
        {
            c->tries += 1;
            if (exceeded && c->tries < sp.max_tries) { c->mode = MODE_RETRY; c->dt_try = c->dt * factor; return; }
        }
    }
    else   // MODE_FINAL (or a committed proposal): accepted
    {
        c->last_max_error = E;
        const int h = c->hist_pos;
        // error of the accepted step before this one (1 before any)
        const int hp = (h + HIST - 1) % HIST;
        const double e_prev = c->hist_dt[hp] > 0 ? c->hist_err[hp] : 1.0;
        const double dt_accepted = c->dt;
        c->hist_dt[h] = c->dt;
        c->hist_err[h] = E;
        c->hist_acc[h] = c->first_passed;
        c->hist_pos = (h + 1) % HIST;
        c->since_div = c->n_divide > 0 ? 0 : c->since_div + 1;
        c->cell_steps += c->n;
        c->t += c->dt;
        c->iter += 1;
        c->iterations += 1;
        // a frame is due when the time has just passed a multiple of dt_write
        // (simulation.hpp:2025-2028)
        if (c->dt_write > 0)
        {
            const double t_old_factor = fmod(c->t - c->dt + 1e-12, c->dt_write);
            const double t_new_factor = fmod(c->t + 1e-12, c->dt_write);
            if (t_old_factor > t_new_factor) c->frame_due = 1;
        }
        if (sp.pi)
        {
            // the PI proposal for the next step: dt 0.9 E^(-0.7/k) E_prev^(0.4/k), k the error
            // order + 1 (Gustafsson's PI rule with the parameters of Hairer & Wanner, Solving
            // ODEs II, sec. IV.2), the factor held to [0.2, 10], dt to [min, max] step size
            double f = 0.9 * pow(1.0 / E, 0.7 * sp.inv_q1) * pow(e_prev, 0.4 * sp.inv_q1);
            if (f >= 10) f = 10;
            else if (f < 0.2) f = 0.2;
            double next = dt_accepted * f;
            if (next < sp.min_stepsize) next = sp.min_stepsize;
            else if (next > sp.max_stepsize) next = sp.max_stepsize;
            c->dt = next;
        }
        c->mode = MODE_TRIAL;
        c->tries = 0;
        c->attempt = 0;
        return;
    }
    // clamp and schedule the final re-run (simulation.hpp:1752-1760)
    double factor = c->factor;
    if (c->dt * factor < sp.min_stepsize) factor = sp.min_stepsize / c->dt;
    else if (c->dt * factor > sp.max_stepsize) factor = sp.max_stepsize / c->dt;
    c->dt *= factor;
    c->dt_try = c->dt;
    c->mode = MODE_FINAL;
}

// friction: the force of cell i at stage st, f0 minus the change of the dE/dq shares of its
// candidate contacts whose planar decision at this stage differs from the one at y0; each
// share enters as the pair sum does, (v, s v) from a lower entry, (-v, -t v) from a partner's
__device__ __forceinline__ void friction_stage_force(const PairGather& pg, int i, int st, const double f0[6],
                                                     double fs[6])
{
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int le = pg.lower_end[i], r1 = pg.row_ptr[i + 1];
    for (int e = pg.row_ptr[i]; e < r1; ++e)
    {
        if (!((pg.fmask[e] >> st) & 1)) continue;
        const double4 dv = pg.fbuf[e];
        const double w = pg.jbuf[e].w;
        const double sg = e < le ? 1.0 : -1.0;
        acc[0] += sg * dv.x; acc[1] += sg * dv.y; acc[2] += sg * dv.z;
        acc[3] += sg * w * dv.x; acc[4] += sg * w * dv.y; acc[5] += sg * w * dv.z;
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) fs[c] = f0[c] - acc[c];
}

// KIND: MODE_TRIAL / MODE_RETRY / MODE_FINAL inside the loop, 3 = API evaluation.
// Without noise the stage-0 velocity k0 = f(y0) is the same for every attempt of an
// iteration (y0 and the pair forces do not change), so the trial stores it in k0buf
// and the retries and the final attempt read it back.
// Learned controller: the trial (the network's proposal) writes its state in place
// and first copies y0 (with l in the gamma slot) and the stored velocity to
// geom_c / vel_c; a proposal that passes the error test closes the step in the
// trial's last block, one that fails continues with retries and a final attempt
// that read y0 back from that copy.
// use_cond bit 0: `cond` is the retry WHILE node's handle; bit 1: `cond_run` is the
// handle of the IF node around the final attempt (0 after a committed proposal).
// Launch bounds: six blocks per SM (85 registers) for the 2- and 4-stage tableaux, the
// fastest measured for the 100k-cell step (three for their friction trial pass, which
// would spill at six); no bound for the 6- and 7-stage ones, which spill below ~130.
// V: 0 FP64; 1 mixed precision; 2 FP64 with cell-cell friction, whose candidate contacts
// add, at each stage whose planar decision differs from the one at y0, the recorded change
// of their shares; 3 the friction trial pass, which runs only the stages of the cells with
// candidate contacts and records their stage states (z, n_z) for the decision check, with
// no other effect.
template <int S, int KIND, bool NOISE, int DIM, int V>
__global__ void __launch_bounds__(AT_T, (S <= 4 ? (V == 3 ? 3 : 6) : 1)) k_attempt(Geom* geom, Vel* vel, Phys* phys, const Gen6* fcc,
                                                 Ctrl* ctrl, StepParams sp, Geom* geom_c, Vel* vel_c,
                                                 Gen6* err_out, Gen6* k0buf, double eval_dt, int eval_attempt,
                                                 unsigned long long cond, int use_cond, PairGather pg,
                                                 unsigned long long cond_run)
{
    constexpr bool F32 = V == 1, FRIC = V >= 2, DRY = V == 3;
    __shared__ double sh_max[AT_T / 32], sh_drift[AT_T / 32];
    __shared__ double4 sh_stat[AT_T / 32];
    __shared__ bool last;
    if (DRY && (!ctrl->fr_pending || (KIND != 3 && ctrl->halted))) return;
    if (KIND != 3 && ctrl->halted)
    {
        // a halted context takes no step: stop an enclosing WHILE node
        if ((use_cond & 1) && (KIND == MODE_TRIAL || KIND == MODE_RETRY) && blockIdx.x == 0 && threadIdx.x == 0)
            cudaGraphSetConditional((cudaGraphConditionalHandle)cond, 0u);
        if ((use_cond & 2) && KIND == MODE_TRIAL && blockIdx.x == 0 && threadIdx.x == 0)
            cudaGraphSetConditional((cudaGraphConditionalHandle)cond_run, 0u);
        return;
    }
    const int n = ctrl->n;
    const int n_order = (KIND != 3 && sp.order) ? ctrl->n_order : 0;
    const int mode = ctrl->mode;
    const int iter = ctrl->iter;
    // the learned and PI controllers propose (and test) a step every iteration
    const bool trial_ran = sp.propose || (iter % sp.iter_update_stepsize == 0);
    // k0 is shared across attempts only under the reference controller: a passing
    // proposal needs no second attempt, so it does not store k0 or the total pair force
    const bool share_k0 = !NOISE && !sp.propose;
    double dt;
    int attempt;
    bool load_k0 = false, store_k0 = false;
    if (KIND == MODE_TRIAL)
    {
        if (!trial_ran) return;   // no step-size update this iteration: FINAL runs at dt
        dt = ctrl->dt; attempt = 0; store_k0 = share_k0;
    }
    else if (KIND == MODE_RETRY)
    {
        if (mode != MODE_RETRY)
        {
            // no retry pending: make sure an enclosing WHILE node stops
            if ((use_cond & 1) && blockIdx.x == 0 && threadIdx.x == 0)
                cudaGraphSetConditional((cudaGraphConditionalHandle)cond, 0u);
            return;
        }
        dt = ctrl->dt_try; attempt = ctrl->attempt; load_k0 = share_k0;
    }
    else if (KIND == MODE_FINAL)
    {
        dt = (mode == MODE_FINAL) ? ctrl->dt_try : ctrl->dt;
        attempt = (mode == MODE_FINAL) ? ctrl->attempt : 0;
        load_k0 = share_k0 && trial_ran;
    }
    else { dt = eval_dt; attempt = eval_attempt; }
    // the step was closed by a proposal that passed the error test
    if (KIND == MODE_FINAL && mode == MODE_COMMIT) return;
    const bool commit = false;
    // a proposal (learned or PI) advances the state in place; the attempts after a failed
    // proposal start from the copy of y0 it kept
    const bool in_place = !DRY && (KIND == MODE_TRIAL) && sp.propose;
    const bool from_backup = (KIND == MODE_RETRY || KIND == MODE_FINAL) && sp.propose;
    if (DRY) store_k0 = false;
    // friction: stages whose planar decisions differ from those at y0 somewhere
    const bool flips = FRIC && ctrl->fr_nflip > 0;

    // the first attempt of an iteration sums the cell's pair shares (pg.fused); under
    // the reference controller the trial writes the total back for the rest, under the
    // proposing ones every attempt sums them
    const bool do_gather = pg.fused && !commit &&
                           (KIND == MODE_TRIAL || (KIND == MODE_FINAL && !trial_ran) || sp.propose);
    double local_max = 0.0;
    bool bad = false;
    double st_vmax = 0.0, st_v2 = 0.0, st_g = 0.0, st_near = 0.0;
    // motion bound of each new segment: |dr| + h' |dn| + |dh| (a Hausdorff bound)
    double local_drift = 0.0;
    // one cell per thread: the grid covers the capacity (attempt_blocks); thread t takes
    // the t-th cell of the attempt order (cells appended after the order was made, in
    // index order).  The body is a do-while(false) block so that `continue` leaves it.
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) do
    {
        const int i = t < n_order ? sp.order[t] : t;
        if (DRY)
        {
            // only cells with a candidate contact have stage states to report
            bool any = false;
            for (int e = pg.row_ptr[i]; e < pg.row_ptr[i + 1] && !any; ++e) any = (pg.fmask[e] & FR_CAND) != 0;
            if (!any) continue;
        }
        const Geom g = load_geom(from_backup ? geom_c : geom, i);
        const Vel* vprev = (from_backup ? vel_c : vel) + i;
        const double y0[6] = {g.rx, g.ry, g.rz, g.nx, g.ny, g.nz};
        // non-finite coordinates (the reference's DEBUG_CHECK_CELL_COORDINATES_NAN,
        // simulation.hpp:1803-1821): a position alone enters no velocity, so its error
        // norm would stay finite
#pragma unroll
        for (int c = 0; c < 6; ++c) if (!isfinite(y0[c])) bad = true;
        const double l = from_backup ? g.gamma : phys[i].l;
        const double eta0 = phys[i].eta0, eta1 = phys[i].eta1, sigma0 = phys[i].sigma0;
        if (in_place)
        {
            Geom b = g;
            b.gamma = l;
            geom_c[i] = b;
            vel_c[i] = vel[i];
        }
        const bool a2 = y0[5] < sp.mp.nz_threshold;
        Gen6 cc;
        if (do_gather)
        {
            cc = pg.fused == 3 ? sum_row_shares(pg.row_ptr, pg.lower_end, reinterpret_cast<const float4*>(pg.jbuf), i)
               : pg.fused == 2 ? sum_row_shares(pg.row_ptr, pg.lower_end, pg.jbuf, i)
                               : gather_pair_force(fcc, pg.row_ptr, pg.lower_end, pg.jbuf, i);
            if (KIND == MODE_TRIAL && !sp.propose && !DRY) pg.fcc_w[i] = cc;
        }
        else cc = (KIND == MODE_TRIAL) ? fcc[i] : load_gen6(fcc, i);
        double f0[6];
        double nz2[4] = {0.0, 0.0, 0.0, 0.0};
        if constexpr (DIM == 2)
        {
            if (NOISE) noise_2d(sp, iter, attempt, i, nz2);
        }
        else base_force<NOISE>(sp, cc, iter, attempt, i, f0);
        double k[S][6];
        if (load_k0)
        {
            const double2* kp = reinterpret_cast<const double2*>(k0buf + i);
            double2 a = kp[0], b = kp[1], c = kp[2];
            k[0][0] = a.x; k[0][1] = a.y; k[0][2] = b.x; k[0][3] = b.y; k[0][4] = c.x; k[0][5] = c.y;
        }
        else
        {
            if constexpr (DIM == 2) velocity_2d(sp, y0, l, eta0, eta1, cc, nz2, k[0]);
            else cell_velocity_p<F32>(sp, a2, y0, l, g.h, eta0, eta1, sigma0, vprev, f0, k[0]);
            if (store_k0)
            {
                double2* kp = reinterpret_cast<double2*>(k0buf + i);
                kp[0] = make_double2(k[0][0], k[0][1]);
                kp[1] = make_double2(k[0][2], k[0][3]);
                kp[2] = make_double2(k[0][4], k[0][5]);
            }
        }
#pragma unroll
        for (int st = 1; st < S; ++st)
        {
            double y[6];
#pragma unroll
            for (int c = 0; c < 6; ++c)
            {
                double m = 0.0;
#pragma unroll
                for (int j = 0; j < st; ++j) m += k[j][c] * sp.A[st][j];
                y[c] = y0[c] + m * dt;
            }
            normalize_n(y);
            if constexpr (DIM == 2) velocity_2d(sp, y, l, eta0, eta1, cc, nz2, k[st]);
            else if constexpr (FRIC)
            {
                if (DRY) pg.ystage[(size_t)st * pg.ystage_ld + i] = make_double2(y[2], y[5]);
                if (flips)
                {
                    double fs[6];
                    friction_stage_force(pg, i, st, f0, fs);
                    cell_velocity_p<false>(sp, a2, y, l, g.h, eta0, eta1, sigma0, vprev, fs, k[st]);
                }
                else cell_velocity_p<false>(sp, a2, y, l, g.h, eta0, eta1, sigma0, vprev, f0, k[st]);
            }
            else cell_velocity_p<F32>(sp, a2, y, l, g.h, eta0, eta1, sigma0, vprev, f0, k[st]);
        }
        if (DRY)
        {
            pg.ystage[i] = make_double2(y0[2], y0[5]);
            continue;
        }
        double vf1[6], d1[6];
#pragma unroll
        for (int c = 0; c < 6; ++c)
        {
            double s1 = 0.0, s2 = 0.0;
#pragma unroll
            for (int st = 0; st < S; ++st) { s1 += k[st][c] * sp.b[st]; s2 += k[st][c] * sp.bs[st]; }
            vf1[c] = s1;
            d1[c] = s1 * dt;
            double err = d1[c] - s2 * dt;
            double scaled = err / (sp.tol * (1.0 + fabs(y0[c])));
            if (isnan(scaled) || isinf(scaled)) bad = true;
            local_max = fmax(local_max, scaled);
            if (KIND == 3 && err_out) err_out[i].f[c] = err;
        }
        if (KIND == MODE_FINAL || KIND == 3 || in_place)
        {
            double y1[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) y1[c] = y0[c] + d1[c];
            normalize_n(y1);
            Geom go = g;
            go.rx = y1[0]; go.ry = y1[1]; go.rz = y1[2]; go.nx = y1[3]; go.ny = y1[4]; go.nz = y1[5];
            Vel vo;
#pragma unroll
            for (int c = 0; c < 6; ++c) vo.v[c] = vf1[c];
            if (KIND == MODE_FINAL || in_place)
            {
                // growCells (growth.hpp:51-57) fused with the accepted step
                const double g_rate = phys[i].growth;
                double lg = l + g_rate * (4 * sp.mp.R / 3 + l) * dt;
                go.h = lg / 2;
                {
                    const double ax = go.rx - g.rx, ay = go.ry - g.ry, az = go.rz - g.rz;
                    const double bx = go.nx - g.nx, by = go.ny - g.ny, bz = go.nz - g.nz;
                    local_drift = fmax(local_drift, sqrt(ax * ax + ay * ay + az * az)
                                                        + go.h * sqrt(bx * bx + by * by + bz * bz)
                                                        + fabs(go.h - g.h));
                }
                if (from_backup) go.gamma = geom[i].gamma;   // the copy holds l in that slot
                phys[i].l = lg;
                geom[i] = go;
                vel[i] = vo;
                if (sp.stats_on)
                {
                    const double v2 = vf1[0] * vf1[0] + vf1[1] * vf1[1] + vf1[2] * vf1[2];
                    st_vmax = fmax(st_vmax, sqrt(v2));
                    st_v2 += v2;
                    st_g += g_rate;
                    st_near += (lg > sp.near_div_length) ? 1.0 : 0.0;
                }
            }
            else
            {
                geom_c[i] = go;
                vel_c[i] = vo;
            }
        }
    } while (false);
    if (DRY) return;
    if ((KIND == MODE_FINAL || in_place) && sp.stats_on)
    {
        // per-block partials of the step-size features, summed in block order later
        st_vmax = warp_max(st_vmax);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            st_v2 += __shfl_xor_sync(0xffffffffu, st_v2, off);
            st_g += __shfl_xor_sync(0xffffffffu, st_g, off);
            st_near += __shfl_xor_sync(0xffffffffu, st_near, off);
        }
        if ((threadIdx.x & 31) == 0) sh_stat[threadIdx.x >> 5] = make_double4(st_vmax, st_v2, st_g, st_near);
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double4 a = sh_stat[0];
            for (int w = 1; w < AT_T / 32; ++w)
            {
                const double4 b = sh_stat[w];
                a.x = fmax(a.x, b.x); a.y += b.y; a.z += b.z; a.w += b.w;
            }
            // the last block sums the partials in block order (no contended atomics)
            sp.stat_part[blockIdx.x] = a;
        }
    }
    if (KIND == MODE_FINAL || in_place)
    {
        local_drift = warp_max(local_drift);
        if ((threadIdx.x & 31) == 0) sh_drift[threadIdx.x >> 5] = local_drift;
    }
    // block max of the scaled error, floored at min_error (simulation.hpp:1703)
    local_max = fmax(local_max, sp.min_error);
    if (bad) local_max = __longlong_as_double(0x7ff0000000000000ll);
    local_max = warp_max(local_max);
    if ((threadIdx.x & 31) == 0) sh_max[threadIdx.x >> 5] = local_max;
    // any thread of the block that met a non-finite value reports it
    const int block_bad = __syncthreads_or(bad ? 1 : 0);
    if (threadIdx.x == 0)
    {
        double m = sh_max[0];
        for (int w = 1; w < AT_T / 32; ++w) m = fmax(m, sh_max[w]);
        unsigned long long bits = (unsigned long long)__double_as_longlong(m);
        if (block_bad) atomicOr(&ctrl->status, (int)ST_NAN);
        if (KIND == MODE_FINAL || in_place)
        {
            double dm = sh_drift[0];
            for (int w = 1; w < AT_T / 32; ++w) dm = fmax(dm, sh_drift[w]);
            if (dm > 0) atomicMax(&ctrl->drift_bits, (unsigned long long)__double_as_longlong(dm));
        }
        if (KIND == 3) { atomicMax(&ctrl->eval_err_bits, bits); last = false; }
        else
        {
            atomicMax(&ctrl->err_bits, bits);
            __threadfence();
            unsigned int done = atomicAdd(&ctrl->blocks_done, 1u);
            last = (done == gridDim.x - 1);
        }
    }
    __syncthreads();
    if ((KIND == MODE_FINAL || in_place) && sp.stats_on && last)
    {
        // step-size features of the accepted step (a failed proposal's are replaced
        // by the final attempt's): every block's partial, in block order
        __threadfence();
        double4 a = make_double4(0.0, 0.0, 0.0, 0.0);
        for (int b = threadIdx.x; b < gridDim.x; b += AT_T)
        {
            const double2* q = reinterpret_cast<const double2*>(sp.stat_part + b);
            const double2 p0 = __ldcg(q), p1 = __ldcg(q + 1);
            a.x = fmax(a.x, p0.x); a.y += p0.y; a.z += p1.x; a.w += p1.y;
        }
        a.x = warp_max(a.x);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            a.y += __shfl_xor_sync(0xffffffffu, a.y, off);
            a.z += __shfl_xor_sync(0xffffffffu, a.z, off);
            a.w += __shfl_xor_sync(0xffffffffu, a.w, off);
        }
        __syncthreads();
        if ((threadIdx.x & 31) == 0) sh_stat[threadIdx.x >> 5] = a;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double4 t = sh_stat[0];
            for (int w = 1; w < AT_T / 32; ++w)
            {
                const double4 b = sh_stat[w];
                t.x = fmax(t.x, b.x); t.y += b.y; t.z += b.z; t.w += b.w;
            }
            ctrl->st_vmax_bits = (unsigned long long)__double_as_longlong(t.x);
            ctrl->st_v2_fx = (unsigned long long)llrint(ldexp(t.y, STAT_V2_SHIFT));
            ctrl->st_g_fx = (unsigned long long)llrint(ldexp(fmax(t.z, 0.0), STAT_G_SHIFT));
            ctrl->st_near_div = (unsigned long long)t.w;
        }
    }
    if (KIND != 3 && last && threadIdx.x == 0)
    {
        __threadfence();
        double E = __longlong_as_double((long long)atomicAdd(&ctrl->err_bits, 0ull));
        E = fmax(E, sp.min_error);
        if (commit) E = ctrl->last_trial_error;
        // motion of the new state, counted once the step is accepted
        const double dm = __longlong_as_double((long long)atomicAdd(&ctrl->drift_bits, 0ull));
        if (KIND == MODE_FINAL) ctrl->drift += dm;
        ctrl->drift_bits = 0ull;
        ctrl->err_bits = 0ull;
        ctrl->blocks_done = 0u;
        controller_finish(ctrl, sp, KIND, E, commit);
        if (in_place && ctrl->mode == MODE_COMMIT)
        {
            // the proposal passed: its state is in place; close the step and leave
            // MODE_COMMIT so that this iteration's final attempt exits at once
            ctrl->drift += dm;
            controller_finish(ctrl, sp, MODE_FINAL, E, true);
            ctrl->mode = MODE_COMMIT;
        }
        // another retry?  (bounded: the controller schedules at most max_tries of them)
        if ((use_cond & 1) && (KIND == MODE_TRIAL || KIND == MODE_RETRY))
            cudaGraphSetConditional((cudaGraphConditionalHandle)cond,
                                    (ctrl->mode == MODE_RETRY && ctrl->tries < sp.max_tries) ? 1u : 0u);
        if ((use_cond & 2) && KIND == MODE_TRIAL)
            cudaGraphSetConditional((cudaGraphConditionalHandle)cond_run, ctrl->mode != MODE_COMMIT ? 1u : 0u);
    }
}

// Frame snapshot, at the end of an iteration: when the accepted step marked a frame,
// every cell's records go to ring slot frames_taken % slots, and the last block
// records the frame's time, iteration, cell count and lineage length.  The loop
// keeps running; the host downloads the slots when it writes the frames.
__global__ void k_frame_snapshot(const Geom* __restrict__ geom, const Vel* __restrict__ vel,
                                 const Phys* __restrict__ phys, Ctrl* ctrl, Geom* snap_geom, Vel* snap_vel,
                                 Phys* snap_phys, FrameInfo* info, int slots, int cap_cells,
                                 const double* __restrict__ feta, double* snap_feta)
{
    __shared__ bool last;
    // frame_due changes only in the last block below, after every block has passed here
    if (!ctrl->frame_due) return;
    const int n = ctrl->n;
    const size_t off = (size_t)(ctrl->frames_taken % slots) * cap_cells;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        snap_geom[off + i] = geom[i];
        snap_vel[off + i] = vel[i];
        snap_phys[off + i] = phys[i];
        if (feta) snap_feta[off + i] = feta[i];
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        last = atomicAdd(&ctrl->frame_blocks, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0)
    {
        FrameInfo f;
        f.t = ctrl->t;
        f.iter = ctrl->iter;
        f.n = n;
        f.n_parents = ctrl->n_parents;
        f.pad = 0;
        info[ctrl->frames_taken % slots] = f;
        ctrl->frames_taken += 1;
        ctrl->frame_due = 0;
        ctrl->frame_blocks = 0u;
    }
}

void launch_frame_snapshot(const Geom* geom, const Vel* vel, const Phys* phys, Ctrl* ctrl, Geom* snap_geom,
                           Vel* snap_vel, Phys* snap_phys, FrameInfo* info, int slots, int cap_cells,
                           cudaStream_t st, const double* feta, double* snap_feta)
{
    const int blocks = max(min(cdiv(cap_cells, 256), 4 * 148), 1);
    k_frame_snapshot<<<blocks, 256, 0, st>>>(geom, vel, phys, ctrl, snap_geom, snap_vel, snap_phys, info, slots,
                                             cap_cells, feta, snap_feta);
}

// Attempt order (3-D): the cells whose velocity takes the full surface solve
// (area integrals, mechanics.hpp:2254-2309) first, then the others, each group in
// index order, so that the warps of an attempt mostly run one of the three
// branches of getVelocities (mechanics.hpp:2011-2347) instead of all of them.
// Made at every neighbor rebuild from the cells of that moment; a cell that
// changes branch before the next rebuild costs only divergence.  The order
// changes no per-cell result.
__global__ void k_attempt_class(const Geom* __restrict__ geom, const Ctrl* ctrl, MechParams P, int* flag)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const Geom g = load_geom(geom, i);
        const bool a2 = g.nz < P.nz_threshold;
        const bool contact = a2 ? (g.rz < P.R) : ((g.rz - g.h * g.nz < P.R) || (g.rz + g.h * g.nz < P.R));
        flag[i] = (!P.no_surface && !a2 && contact) ? 1 : 0;
    }
}

__global__ void k_attempt_order(Ctrl* ctrl, const int* __restrict__ flag, const int* __restrict__ pos, int* order)
{
    const int n = ctrl->n;
    const int n_full = pos[n];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        order[flag[i] ? pos[i] : n_full + (i - pos[i])] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->n_order = n;
}

void launch_attempt_order(const Geom* geom, Ctrl* ctrl, const MechParams& P, int* flag, int* pos,
                          int* block_sums, int* order, int cap_cells, cudaStream_t st)
{
    const int blocks = max(cdiv(cap_cells, 256), 1);
    k_attempt_class<<<blocks, 256, 0, st>>>(geom, ctrl, P, flag);
    launch_scan(flag, &ctrl->n, pos, block_sums, cap_cells, st);
    k_attempt_order<<<blocks, 256, 0, st>>>(ctrl, flag, pos, order);
}

template <int S, bool NOISE, int DIM, int V>
static void launch_attempt_s(int kind, int blocks, Geom* geom, Vel* vel, Phys* phys, const Gen6* fcc,
                             Ctrl* ctrl, const StepParams& sp, Geom* geom_c, Vel* vel_c, Gen6* err_out,
                             Gen6* k0buf, double eval_dt, int eval_attempt, cudaStream_t st,
                             unsigned long long cond, int use_cond, PairGather pg, unsigned long long cond_run)
{
#define AT_ARGS geom, vel, phys, fcc, ctrl, sp, geom_c, vel_c, err_out, k0buf, eval_dt, eval_attempt, cond, use_cond, pg, cond_run
#define AT_LAUNCH(K) k_attempt<S, K, NOISE, DIM, V><<<blocks, AT_T, 0, st>>>(AT_ARGS);
    switch (kind)
    {
        case MODE_TRIAL: AT_LAUNCH(MODE_TRIAL) break;
        case MODE_RETRY: AT_LAUNCH(MODE_RETRY) break;
        case MODE_FINAL: AT_LAUNCH(MODE_FINAL) break;
        default: AT_LAUNCH(3) break;
    }
#undef AT_LAUNCH
#undef AT_ARGS
}

int attempt_blocks(int cap_cells) { return max(cdiv(cap_cells, AT_T), 1); }

void launch_attempt(int kind, Geom* geom, Vel* vel, Phys* phys, const Gen6* fcc, Ctrl* ctrl,
                    const StepParams& sp, Geom* geom_c, Vel* vel_c, Gen6* err_out, Gen6* k0buf,
                    double eval_dt, int eval_attempt, int cap_cells, cudaStream_t st,
                    unsigned long long cond, int use_cond, PairGather pg, int dims, unsigned long long cond_run)
{
    int blocks = attempt_blocks(cap_cells);
#define AT_CALL(S, NZ, D, F) launch_attempt_s<S, NZ, D, F>(kind, blocks, geom, vel, phys, fcc, ctrl, sp, geom_c, vel_c, err_out, k0buf, eval_dt, eval_attempt, st, cond, use_cond, pg, cond_run)
#define AT_CASE(S, D) case S: \
        if (D == 3 && sp.mixed) { if (sp.noise_on) AT_CALL(S, true, D, (D == 3 ? 1 : 0)); else AT_CALL(S, false, D, (D == 3 ? 1 : 0)); } \
        else if (D == 3 && sp.fric) { if (sp.noise_on) AT_CALL(S, true, D, (D == 3 ? 2 : 0)); else AT_CALL(S, false, D, (D == 3 ? 2 : 0)); } \
        else if (sp.noise_on) AT_CALL(S, true, D, 0); \
        else AT_CALL(S, false, D, 0); \
        break;
    if (dims == 2)
    {
        // the 2-D driver integrates with Bogacki-Shampine 3(2) (2D/include/simulation.hpp:217-228);
        // Heun-Euler is kept for comparison runs
        switch (sp.s)
        {
            AT_CASE(2, 2) AT_CASE(4, 2)
            default: break;
        }
        return;
    }
    switch (sp.s)
    {
        AT_CASE(2, 3) AT_CASE(4, 3) AT_CASE(6, 3) AT_CASE(7, 3)
        default: break;
    }
#undef AT_CASE
#undef AT_CALL
}

// Friction decision check over the candidate pairs of the last pair pass: the planar
// decision of each stage from the two cells' stage states (the contact points
// r + s n of both cells below 1.01 R, mechanics.hpp:1090-1110), compared with the one at
// y0; a pair whose set of differing stages changed is updated in both entries.  The last
// block schedules another trial pass when any pair changed.
__global__ void k_fr_check(Ctrl* ctrl, const int4* __restrict__ pairs, const int* __restrict__ fr_list,
                           const double4* __restrict__ jbuf, const double2* __restrict__ ystage, int ld, int S,
                           int* fmask, double R)
{
    __shared__ bool last;
    if (!ctrl->fr_pending) return;
    const int m = ctrl->fr_ncand;
    const double lim = 1.01 * R;
    int changed = 0, nflip = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x)
    {
        const int4 pr = pairs[fr_list[q]];
        const double s = jbuf[pr.z].w, t = jbuf[pr.w].w;
        const int mk = fmask[pr.z];
        const bool d0 = (mk & FR_D0) != 0;
        int fl = 0;
        for (int st = 1; st < S; ++st)
        {
            const double2 a = ystage[(size_t)st * ld + pr.x], b = ystage[(size_t)st * ld + pr.y];
            const bool flat = __dadd_rn(a.x, __dmul_rn(s, a.y)) < lim && __dadd_rn(b.x, __dmul_rn(t, b.y)) < lim;
            if (flat != d0) fl |= 1 << st;
        }
        if (fl != (mk & FR_FLIPS))
        {
            fmask[pr.z] = (mk & ~FR_FLIPS) | fl;
            fmask[pr.w] = (fmask[pr.w] & ~FR_FLIPS) | fl;
            changed = 1;
        }
        nflip += fl != 0;
    }
    changed = __syncthreads_or(changed);
    if (nflip) atomicAdd(&ctrl->fr_nflip_next, nflip);
    if (threadIdx.x == 0)
    {
        if (changed) atomicOr(&ctrl->fr_changed, 1);
        __threadfence();
        last = atomicAdd(&ctrl->fr_blocks, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0)
    {
        __threadfence();
        ctrl->fr_nflip = atomicAdd(&ctrl->fr_nflip_next, 0);
        ctrl->fr_nflip_next = 0;
        ctrl->fr_pending = atomicAdd(&ctrl->fr_changed, 0);
        ctrl->fr_changed = 0;
        ctrl->fr_blocks = 0u;
    }
}

__global__ void k_fr_arm(Ctrl* ctrl) { ctrl->fr_pending = ctrl->fr_ncand > 0 && !ctrl->halted; }

template <int S, int KIND, bool NOISE>
static void launch_fr_rounds_s(Geom* geom, Vel* vel, Phys* phys, const Gen6* fcc, Ctrl* ctrl, const StepParams& sp,
                               Geom* geom_c, Vel* vel_c, Gen6* k0buf, double eval_dt, int eval_attempt, int blocks,
                               cudaStream_t st, PairGather pg, const int4* pairs, const int* fr_list, int* fmask,
                               double R, int check_blocks)
{
    k_fr_arm<<<1, 1, 0, st>>>(ctrl);
    for (int r = 1; r < S; ++r)
    {
        k_attempt<S, KIND, NOISE, 3, 3><<<blocks, AT_T, 0, st>>>(geom, vel, phys, fcc, ctrl, sp, geom_c, vel_c, nullptr, k0buf, eval_dt,
                                 eval_attempt, 0ull, 0, pg, 0ull);
        k_fr_check<<<check_blocks, 256, 0, st>>>(ctrl, pairs, fr_list, pg.jbuf, pg.ystage, pg.ystage_ld, S, fmask, R);
    }
}

void launch_friction_rounds(int kind, Geom* geom, Vel* vel, Phys* phys, const Gen6* fcc, Ctrl* ctrl,
                            const StepParams& sp, Geom* geom_c, Vel* vel_c, Gen6* k0buf, double eval_dt,
                            int eval_attempt, int cap_cells, cudaStream_t st, PairGather pg, const int4* pairs,
                            const int* fr_list, int* fmask, double R)
{
    const int blocks = attempt_blocks(cap_cells);
    const int cb = 148 * 2;
#define FR_K(S, K) { if (sp.noise_on) launch_fr_rounds_s<S, K, true>(geom, vel, phys, fcc, ctrl, sp, geom_c, vel_c, k0buf, eval_dt, eval_attempt, blocks, st, pg, pairs, fr_list, fmask, R, cb); \
                     else launch_fr_rounds_s<S, K, false>(geom, vel, phys, fcc, ctrl, sp, geom_c, vel_c, k0buf, eval_dt, eval_attempt, blocks, st, pg, pairs, fr_list, fmask, R, cb); }
#define FR_S(S) case S: \
        switch (kind) { case MODE_TRIAL: FR_K(S, MODE_TRIAL) break; case MODE_RETRY: FR_K(S, MODE_RETRY) break; \
                        case MODE_FINAL: FR_K(S, MODE_FINAL) break; default: FR_K(S, 3) break; } \
        break;
    switch (sp.s)
    {
        FR_S(2) FR_S(4) FR_S(6) FR_S(7)
        default: break;
    }
#undef FR_S
#undef FR_K
}

__global__ void k_velocities_2d(const Geom* __restrict__ geom, const Phys* __restrict__ phys,
                                const Gen6* __restrict__ fcc, const Ctrl* ctrl, StepParams sp, Gen6* v_out)
{
    const int n = ctrl->n;
    const double nz[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const Geom g = load_geom(geom, i);
        const double y[6] = {g.rx, g.ry, g.rz, g.nx, g.ny, g.nz};
        const Phys ph = phys[i];
        Gen6 out;
        velocity_2d(sp, y, ph.l, ph.eta0, ph.eta1, load_gen6(fcc, i), nz, out.f);
        v_out[i] = out;
    }
}

__global__ void k_velocities(const Geom* __restrict__ geom, const Vel* __restrict__ vel,
                             const Phys* __restrict__ phys, const Gen6* __restrict__ fcc, const Ctrl* ctrl,
                             StepParams sp, Gen6* v_out)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const Geom g = load_geom(geom, i);
        const double y[6] = {g.rx, g.ry, g.rz, g.nx, g.ny, g.nz};
        const bool a2 = y[5] < sp.mp.nz_threshold;
        double f0[6];
        base_force<false>(sp, load_gen6(fcc, i), 0, 0, i, f0);
        Gen6 out;
        const Phys ph = phys[i];
        if (sp.mixed) cell_velocity_f32(sp, a2, y, ph.l, g.h, ph.eta0, ph.eta1, ph.sigma0, vel + i, f0, out.f);
        else cell_velocity(sp, a2, y, ph.l, g.h, ph.eta0, ph.eta1, ph.sigma0, vel + i, f0, out.f);
        v_out[i] = out;
    }
}

void launch_velocities(const Geom* geom, const Vel* vel, const Phys* phys, const Gen6* fcc,
                       const Ctrl* ctrl, const StepParams& sp, Gen6* v_out, int cap_cells,
                       cudaStream_t st, int dims)
{
    if (dims == 2)
    {
        k_velocities_2d<<<max(cdiv(cap_cells, 128), 1), 128, 0, st>>>(geom, phys, fcc, ctrl, sp, v_out);
        return;
    }
    k_velocities<<<max(cdiv(cap_cells, 128), 1), 128, 0, st>>>(geom, vel, phys, fcc, ctrl, sp, v_out);
}

// growCells (growth.hpp:51-57)
__global__ void k_grow(Geom* geom, Phys* phys, const Ctrl* ctrl, double R, double dt)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        double l = phys[i].l;
        l += phys[i].growth * (4 * R / 3 + l) * dt;
        phys[i].l = l;
        geom[i].h = l / 2;
    }
}

void launch_grow(Geom* geom, Phys* phys, const Ctrl* ctrl, double R, double dt, int cap_cells,
                 cudaStream_t st)
{
    k_grow<<<max(cdiv(cap_cells, 256), 1), 256, 0, st>>>(geom, phys, ctrl, R, dt);
}

// ---------------------------------------------------------------------------
// Neighbor table in the reference's row order (i ascending, j < i ascending)
// ---------------------------------------------------------------------------
__global__ void k_count_lower(const Ctrl* ctrl, const int* row_ptr, const int* col, int* cnt)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        int c = 0;
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) c += col[k] < i;
        cnt[i] = c;
    }
}

void launch_count_lower(const Ctrl* ctrl, const int* row_ptr, const int* col, int* cnt,
                        int cap_cells, cudaStream_t st)
{
    k_count_lower<<<max(cdiv(cap_cells, 256), 1), 256, 0, st>>>(ctrl, row_ptr, col, cnt);
}

// 3-D rows (i, j, dx, dy, dz, si, sj); 2-D rows (i, j, dx, dy, si, sj)
__global__ void k_table_rows(const Ctrl* ctrl, const int* row_ptr, const int* col, const int* pos,
                             const Geom* __restrict__ geom, double* out, int ld, int dims)
{
    const int n = ctrl->n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        int p = pos[i];
        Geom gi = load_geom(geom, i);
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
        {
            int j = col[k];
            if (j >= i) continue;
            Dist d = dist_geom(gi, load_geom(geom, j));
            out[p] = i; out[(size_t)ld + p] = j;
            out[(size_t)2 * ld + p] = d.dx; out[(size_t)3 * ld + p] = d.dy;
            if (dims == 2)
            {
                out[(size_t)4 * ld + p] = d.s; out[(size_t)5 * ld + p] = d.t;
            }
            else
            {
                out[(size_t)4 * ld + p] = d.dz;
                out[(size_t)5 * ld + p] = d.s; out[(size_t)6 * ld + p] = d.t;
            }
            ++p;
        }
    }
}

void launch_table_rows(const Ctrl* ctrl, const int* row_ptr, const int* col, const int* pos,
                       const Geom* geom, double* out, int ld, int cap_cells, cudaStream_t st, int dims)
{
    k_table_rows<<<max(cdiv(cap_cells, 128), 1), 128, 0, st>>>(ctrl, row_ptr, col, pos, geom, out, ld, dims);
}

}   // namespace abm
