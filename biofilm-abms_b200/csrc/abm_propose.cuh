// Step-size proposal of the learned controller, shared by the network kernels
// (abm_mlp.cu) and the pair pass (abm_kernels.cu), which runs it in one of its blocks.
// BF16 operands, FP32 accumulation on the tensor cores (mma.sync m16n8k16).
#pragma once
#include <cuda_bf16.h>
#include "abm_kernels.cuh"

namespace abm {

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                 "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------------------
// Inside the loop (after the pair force, before the first attempt).
// Features, in order:
//   0       ln(n) / 10
//   1       log10(max |v_r| + 1e-12) / 4     (velocities of the last accepted step)
//   2       log10(rms |v_r| + 1e-12) / 4
//   3       max overlap / (2 (R - Rcell))    (the previous iteration's pair pass)
//   4..11   log10(dt / max_stepsize) of the last 8 accepted steps, newest first
//   12..19  log10(scaled error) / 10 of those steps
//   20..27  1 if that step's first attempt passed the error test
//   28      mean growth rate (1/h)
//   29      fraction of cells longer than 0.9 Ldiv
//   30      log10(1 + cells dividing this iteration)
//   31      ln(1 + iterations since the last division) / 5
// Before any history exists the slots repeat the current dt with error 1, passed.
//
// The proposal is ln(dt / dt_prev) = clamp(b + y, ln 0.2, ln 10) with y the network
// output and b the error-model baseline of the reference controller's factor
// (simulation.hpp:1710): b = ln 0.9 - ln(E_last) / (q + 1), E_last the scaled error
// of the last accepted step, read from feature 12 so that training (which
// subtracts the logged b from its targets) and inference see the same value.  The
// network learns a correction to the error model; where it has nothing to add,
// the proposal is the classical one-step controller, which keeps dt stable.
// After a failed first attempt among the last 8 steps the correction is capped at 0.
// ---------------------------------------------------------------------------
// One 8-unit tile of a hidden layer for row 0 (the other 15 rows of the MMA are
// zero): warp `j` computes units 8j..8j+7 from the layer input in shared memory,
// with the same MMA sequence (k-steps in order) as mlp_tile_forward_regs.
template <int K>
__device__ __forceinline__ void row0_tile(const float* __restrict__ W, int w_off, int b_off, const float* in,
                                          float* out, int j)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    const float* wr = W + w_off + (8 * j + g) * K;
#pragma unroll
    for (int kk = 0; kk < K / 16; ++kk)
    {
        const int k0 = 16 * kk + 2 * t;
        const uint32_t a0 = g == 0 ? pack_bf16(in[k0], in[k0 + 1]) : 0u;
        const uint32_t a2 = g == 0 ? pack_bf16(in[k0 + 8], in[k0 + 9]) : 0u;
        mma_bf16(c, a0, 0u, a2, 0u, pack_bf16(wr[k0], wr[k0 + 1]), pack_bf16(wr[k0 + 8], wr[k0 + 9]));
    }
    if (g == 0)
    {
        out[8 * j + 2 * t] = fmaxf(c[0] + W[b_off + 8 * j + 2 * t], 0.f);
        out[8 * j + 2 * t + 1] = fmaxf(c[1] + W[b_off + 8 * j + 2 * t + 1], 0.f);
    }
}

// One block of 8 warps (blockDim.x == 256): features, then layer 1 and layer 2 one
// 8-unit tile per warp, then the output unit on warp 0 (bit-identical to
// mlp_tile_forward_regs for row 0).  Runs in one block of the pair pass, beside the
// blocks that compute the pairs: nothing it reads is written during that pass.
static __device__ __forceinline__ void mlp_propose_block(Ctrl* ctrl, const StepParams& sp, const float* __restrict__ W)
{
    __shared__ float feat[MLP_IN], h1[MLP_H], h2[MLP_H];
    __shared__ float sh_base;
    __shared__ int sh_fail;
    if (ctrl->halted) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int n = ctrl->n;
    const double inv_n = 1.0 / (double)max(n, 1);
    // The step statistics, one feature per thread (the FP64 logarithms run side by
    // side rather than one after another): the sums of the last accepted step (final
    // attempt or accepted proposal) and the previous pass's overlap maximum, each read
    // and then reset by the thread that uses it.
    switch (tid)
    {
    case 0: feat[0] = (float)(log((double)max(n, 1)) / 10.0); break;
    case 1:
    {
        const double vmax = __longlong_as_double((long long)ctrl->st_vmax_bits);
        ctrl->st_vmax_bits = 0ull;
        feat[1] = (float)(log10(vmax + 1e-12) / 4.0);
        break;
    }
    case 2:
    {
        const double v2 = ldexp((double)ctrl->st_v2_fx, -STAT_V2_SHIFT);
        ctrl->st_v2_fx = 0ull;
        feat[2] = (float)(log10(sqrt(v2 * inv_n) + 1e-12) / 4.0);
        break;
    }
    case 3:
    {
        // the previous iteration's pass (the other parity), made by its blocks'
        // atomicMax: taken and cleared at L2 for the next iteration's pass
        const double ovl = __longlong_as_double((long long)atomicExch(&ctrl->st_ovl_bits[(ctrl->iter + 1) & 1], 0ull));
        feat[3] = (float)(ovl / (2 * (sp.mp.R - sp.mp.Rcell)));
        break;
    }
    case 4:
    {
        const double gs = ldexp((double)ctrl->st_g_fx, -STAT_G_SHIFT);
        ctrl->st_g_fx = 0ull;
        feat[28] = (float)(gs * inv_n);
        break;
    }
    case 5:
    {
        const double near = (double)ctrl->st_near_div;
        ctrl->st_near_div = 0ull;
        feat[29] = (float)(near * inv_n);
        break;
    }
    case 6: feat[30] = (float)log10(1.0 + (double)ctrl->n_divide); break;
    case 7: feat[31] = (float)(log1p((double)ctrl->since_div) / 5.0); break;
    default: break;
    }
    if (tid >= 32 && tid < 32 + HIST)
    {
        const int k = tid - 32;
        const int slot = (ctrl->hist_pos - 1 - k + 2 * HIST) % HIST;
        const bool have = ctrl->hist_dt[slot] > 0;
        const double hd = have ? ctrl->hist_dt[slot] : ctrl->dt;
        const double he = have ? ctrl->hist_err[slot] : 1.0;
        feat[4 + k] = (float)log10(hd / sp.max_stepsize);
        feat[12 + k] = (float)(log10(fmax(he, 1e-30)) / 10.0);
        feat[20 + k] = have ? (float)ctrl->hist_acc[slot] : 1.f;
    }
    __syncthreads();
    if (tid == 0)
    {
        // the PI rule's ln ratio: ln 0.9 - (0.7 ln E_last - 0.4 ln E_prev) / (q + 1), with
        // ln E = ln(10) * 10 * features 12 and 13 (the last two accepted steps)
        const double lnE_last = (double)(2.302585093f * 10.f * feat[12]);
        const double lnE_prev = (double)(2.302585093f * 10.f * feat[13]);
        sh_base = (float)(log(0.9) - sp.inv_q1 * (0.7 * lnE_last - 0.4 * lnE_prev));
        int fail = 0;
        for (int k = 0; k < HIST; ++k) fail |= feat[20 + k] < 0.5f;
        sh_fail = fail;
    }
    __syncthreads();
    if (sp.log_cap > 0 && wid == 0)
    {
        float* row = sp.log_buf + (size_t)(ctrl->log_rows % sp.log_cap) * MLP_LOG_COLS;
        row[lane] = feat[lane];
        if (lane == 0) { row[36] = sh_base; row[37] = 0.f; row[38] = 0.f; row[39] = 0.f; }
    }
    const double dt_prev = ctrl->dt;
    if (!sp.network)
    {
        if (tid == 0) ctrl->dt_prev = dt_prev;
        return;
    }
    row0_tile<MLP_IN>(W, MLP_OFF_W1, MLP_OFF_B1, feat, h1, wid);
    __syncthreads();
    row0_tile<MLP_H>(W, MLP_OFF_W2, MLP_OFF_B2, h1, h2, wid);
    __syncthreads();
    if (wid != 0) return;
    const int g = lane >> 2, t = lane & 3;
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    const float* w3 = W + MLP_OFF_W3;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
    {
        const int k0 = 16 * kk + 2 * t;
        const uint32_t a0 = g == 0 ? pack_bf16(h2[k0], h2[k0 + 1]) : 0u;
        const uint32_t a2 = g == 0 ? pack_bf16(h2[k0 + 8], h2[k0 + 9]) : 0u;
        const uint32_t b0 = g == 0 ? pack_bf16(w3[k0], w3[k0 + 1]) : 0u;
        const uint32_t b1 = g == 0 ? pack_bf16(w3[k0 + 8], w3[k0 + 9]) : 0u;
        mma_bf16(c, a0, 0u, a2, 0u, b0, b1);
    }
    if (lane == 0)
    {
        float y0 = c[0] + W[MLP_OFF_B3];
        // after a failed first attempt among the last 8 steps the network may only
        // shrink the step: a network that keeps asking for too much cannot make
        // every proposal fail
        if (sh_fail) y0 = fminf(y0, 0.f);
        // ln ratio within the reference controller's factor bounds [0.2, 10]
        // (simulation.hpp:1710-1713), then the step-size bounds (:1752-1757)
        const double r = fmin(fmax((double)(sh_base + y0), log(0.2)), log(10.0));
        ctrl->dt_prev = dt_prev;
        ctrl->dt = fmin(fmax(dt_prev * exp(r), sp.min_stepsize), sp.max_stepsize);
    }
}

}   // namespace abm
