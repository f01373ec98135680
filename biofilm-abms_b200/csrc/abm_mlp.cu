// Step-size network: a 32 -> 64 -> 64 -> 1 ReLU MLP that proposes ln(dt_next / dt)
// from 32 features of the running simulation.  Every product with a weight matrix
// runs on the tensor cores with BF16 operands and FP32 accumulation (mma.sync
// m16n8k16); the FP32 master weights and the Adam moments live in global memory
// and are rounded to BF16 (round to nearest even) each time a kernel loads them.
//
//   k_mlp_forward    batch inference, 16-row tiles per warp
//   k_mlp_grad       loss and gradient of a batch (checked against a CPU restatement)
//   k_mlp_train      mini-batch Adam on a logged data set, one block of 4 warps
//   mlp_propose_block  inside the loop, in one block of the pair pass
//                    (abm_propose.cuh): the features of the iteration -> log row, and
//                    (learned controller) the network's dt
//
// Forward arithmetic is identical in all of them: the same MMA sequence over the
// same BF16 operands, then bias and ReLU in FP32.
#include <algorithm>
#include <cuda_bf16.h>
#include "abm_kernels.cuh"
#include "abm_propose.cuh"

namespace abm {

// ---------------------------------------------------------------------------
// Forward of one 16-row tile with the activations in registers.  Lane l holds
// rows g = l/4 and g + 8, columns 8j + 2t, 8j + 2t + 1 (t = l%4) of every
// 8-column tile j: the accumulator layout of one layer is the A-fragment
// layout of the next.  X(r, k) gives the input; W is the FP32 master layout.
// Returns the outputs of rows g and g + 8 on the lanes with t == 0.
// ---------------------------------------------------------------------------
template <class FX>
__device__ __forceinline__ float2 mlp_tile_forward_regs(const float* __restrict__ W, FX X)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float h1[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j)
    {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        const float* wr = W + MLP_OFF_W1 + (8 * j + g) * MLP_IN;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk)
        {
            const int k0 = 16 * kk + 2 * t;
            mma_bf16(c, pack_bf16(X(g, k0), X(g, k0 + 1)), pack_bf16(X(g + 8, k0), X(g + 8, k0 + 1)),
                     pack_bf16(X(g, k0 + 8), X(g, k0 + 9)), pack_bf16(X(g + 8, k0 + 8), X(g + 8, k0 + 9)),
                     pack_bf16(wr[k0], wr[k0 + 1]), pack_bf16(wr[k0 + 8], wr[k0 + 9]));
        }
        const float b0 = W[MLP_OFF_B1 + 8 * j + 2 * t], b1 = W[MLP_OFF_B1 + 8 * j + 2 * t + 1];
        h1[j][0] = fmaxf(c[0] + b0, 0.f); h1[j][1] = fmaxf(c[1] + b1, 0.f);
        h1[j][2] = fmaxf(c[2] + b0, 0.f); h1[j][3] = fmaxf(c[3] + b1, 0.f);
    }
    uint32_t a1[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
    {
        a1[kk][0] = pack_bf16(h1[2 * kk][0], h1[2 * kk][1]);
        a1[kk][1] = pack_bf16(h1[2 * kk][2], h1[2 * kk][3]);
        a1[kk][2] = pack_bf16(h1[2 * kk + 1][0], h1[2 * kk + 1][1]);
        a1[kk][3] = pack_bf16(h1[2 * kk + 1][2], h1[2 * kk + 1][3]);
    }
    float h2[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j)
    {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        const float* wr = W + MLP_OFF_W2 + (8 * j + g) * MLP_H;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
        {
            const int k0 = 16 * kk + 2 * t;
            mma_bf16(c, a1[kk][0], a1[kk][1], a1[kk][2], a1[kk][3], pack_bf16(wr[k0], wr[k0 + 1]),
                     pack_bf16(wr[k0 + 8], wr[k0 + 9]));
        }
        const float b0 = W[MLP_OFF_B2 + 8 * j + 2 * t], b1 = W[MLP_OFF_B2 + 8 * j + 2 * t + 1];
        h2[j][0] = fmaxf(c[0] + b0, 0.f); h2[j][1] = fmaxf(c[1] + b1, 0.f);
        h2[j][2] = fmaxf(c[2] + b0, 0.f); h2[j][3] = fmaxf(c[3] + b1, 0.f);
    }
    // output layer: one real column (n = 0) of an 8-column tile
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    const float* w3 = W + MLP_OFF_W3;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
    {
        const int k0 = 16 * kk + 2 * t;
        const uint32_t b0 = g == 0 ? pack_bf16(w3[k0], w3[k0 + 1]) : 0u;
        const uint32_t b1 = g == 0 ? pack_bf16(w3[k0 + 8], w3[k0 + 9]) : 0u;
        mma_bf16(c, pack_bf16(h2[2 * kk][0], h2[2 * kk][1]), pack_bf16(h2[2 * kk][2], h2[2 * kk][3]),
                 pack_bf16(h2[2 * kk + 1][0], h2[2 * kk + 1][1]), pack_bf16(h2[2 * kk + 1][2], h2[2 * kk + 1][3]),
                 b0, b1);
    }
    // lanes with t == 0 hold column 0 of rows g (c[0]) and g + 8 (c[2])
    const float b3 = W[MLP_OFF_B3];
    return make_float2(c[0] + b3, c[2] + b3);
}

// ---------------------------------------------------------------------------
// Shared-memory warp GEMM for training: C[M x N] = A[M x K] B[K x N] through
// accessors, operands rounded to BF16 at load, the same MMA as above.
// ---------------------------------------------------------------------------
template <class FA, class FB, class FS>
__device__ __forceinline__ void warp_gemm(int M, int N, int K, FA a, FB b, FS store)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int mt = 0; mt < M; mt += 16)
        for (int nt = 0; nt < N; nt += 8)
        {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            for (int kt = 0; kt < K; kt += 16)
            {
                const int r0 = mt + g, r1 = mt + g + 8, k0 = kt + 2 * t, k1 = kt + 2 * t + 8, nn = nt + g;
                mma_bf16(c, pack_bf16(a(r0, k0), a(r0, k0 + 1)), pack_bf16(a(r1, k0), a(r1, k0 + 1)),
                         pack_bf16(a(r0, k1), a(r0, k1 + 1)), pack_bf16(a(r1, k1), a(r1, k1 + 1)),
                         pack_bf16(b(k0, nn), b(k0 + 1, nn)), pack_bf16(b(k1, nn), b(k1 + 1, nn)));
            }
            store(mt + g, nt + 2 * t, c[0]);
            store(mt + g, nt + 2 * t + 1, c[1]);
            store(mt + g + 8, nt + 2 * t, c[2]);
            store(mt + g + 8, nt + 2 * t + 1, c[3]);
        }
}

struct WarpTile {
    float X[16 * MLP_IN], T[16], H1[16 * MLP_H], H2[16 * MLP_H], dH[16 * MLP_H], y[16], dY[16];
};

// forward of a staged tile, keeping the hidden activations for the backward pass
__device__ void tile_forward_smem(const float* W, WarpTile& s)
{
    warp_gemm(16, MLP_H, MLP_IN, [&](int r, int k) { return s.X[r * MLP_IN + k]; },
              [&](int k, int n) { return W[MLP_OFF_W1 + n * MLP_IN + k]; },
              [&](int r, int n, float v) { s.H1[r * MLP_H + n] = fmaxf(v + W[MLP_OFF_B1 + n], 0.f); });
    __syncwarp();
    warp_gemm(16, MLP_H, MLP_H, [&](int r, int k) { return s.H1[r * MLP_H + k]; },
              [&](int k, int n) { return W[MLP_OFF_W2 + n * MLP_H + k]; },
              [&](int r, int n, float v) { s.H2[r * MLP_H + n] = fmaxf(v + W[MLP_OFF_B2 + n], 0.f); });
    __syncwarp();
    warp_gemm(16, 8, MLP_H, [&](int r, int k) { return s.H2[r * MLP_H + k]; },
              [&](int k, int n) { return n == 0 ? W[MLP_OFF_W3 + k] : 0.f; },
              [&](int r, int n, float v) { if (n == 0) s.y[r] = v + W[MLP_OFF_B3]; });
    __syncwarp();
}

// gradient of sum_r 0.5 (y_r - t_r)^2 / denom over the tile's `rows` valid rows,
// added into G.  Products with a weight matrix run on the tensor cores like the
// forward; the output layer (one unit) is plain FP32.
__device__ void tile_backward(const float* W, WarpTile& s, int rows, float denom, float* G)
{
    const int lane = threadIdx.x & 31;
    if (lane < 16) s.dY[lane] = lane < rows ? (s.y[lane] - s.T[lane]) / denom : 0.f;
    __syncwarp();
    for (int c = lane; c < MLP_H; c += 32)
    {
        float a = 0.f;
        for (int r = 0; r < 16; ++r) a += s.dY[r] * s.H2[r * MLP_H + c];
        atomicAdd(&G[MLP_OFF_W3 + c], a);
    }
    if (lane == 0)
    {
        float a = 0.f;
        for (int r = 0; r < 16; ++r) a += s.dY[r];
        atomicAdd(&G[MLP_OFF_B3], a);
    }
    // dH2 = dY w3 masked by the ReLU (w3 as the forward saw it, in BF16)
    for (int e = lane; e < 16 * MLP_H; e += 32)
    {
        const int r = e / MLP_H, c = e % MLP_H;
        s.dH[e] = s.H2[e] > 0.f ? s.dY[r] * __bfloat162float(__float2bfloat16_rn(W[MLP_OFF_W3 + c])) : 0.f;
    }
    __syncwarp();
    // dW2[n][k] += sum_r dH2[r][n] H1[r][k]
    warp_gemm(MLP_H, MLP_H, 16, [&](int n, int r) { return s.dH[r * MLP_H + n]; },
              [&](int r, int k) { return s.H1[r * MLP_H + k]; },
              [&](int n, int k, float v) { atomicAdd(&G[MLP_OFF_W2 + n * MLP_H + k], v); });
    for (int c = lane; c < MLP_H; c += 32)
    {
        float a = 0.f;
        for (int r = 0; r < 16; ++r) a += s.dH[r * MLP_H + c];
        atomicAdd(&G[MLP_OFF_B2 + c], a);
    }
    __syncwarp();
    // dH1[r][k] = sum_n dH2[r][n] W2[n][k], masked by the ReLU; written over H2
    warp_gemm(16, MLP_H, MLP_H, [&](int r, int n) { return s.dH[r * MLP_H + n]; },
              [&](int n, int k) { return W[MLP_OFF_W2 + n * MLP_H + k]; },
              [&](int r, int k, float v) { s.H2[r * MLP_H + k] = s.H1[r * MLP_H + k] > 0.f ? v : 0.f; });
    __syncwarp();
    // dW1[n][k] += sum_r dH1[r][n] X[r][k]
    warp_gemm(MLP_H, MLP_IN, 16, [&](int n, int r) { return s.H2[r * MLP_H + n]; },
              [&](int r, int k) { return s.X[r * MLP_IN + k]; },
              [&](int n, int k, float v) { atomicAdd(&G[MLP_OFF_W1 + n * MLP_IN + k], v); });
    for (int c = lane; c < MLP_H; c += 32)
    {
        float a = 0.f;
        for (int r = 0; r < 16; ++r) a += s.H2[r * MLP_H + c];
        atomicAdd(&G[MLP_OFF_B1 + c], a);
    }
    __syncwarp();
}

__device__ void stage_tile(WarpTile& s, const float* X, const float* T, int row0, int n)
{
    const int lane = threadIdx.x & 31;
    for (int e = lane; e < 16 * MLP_IN; e += 32)
    {
        const int r = e / MLP_IN;
        s.X[e] = (row0 + r < n) ? X[(size_t)(row0 + r) * MLP_IN + e % MLP_IN] : 0.f;
    }
    if (lane < 16) s.T[lane] = (T && row0 + lane < n) ? T[row0 + lane] : 0.f;
    __syncwarp();
}

const int MLP_WARPS = 4;

// batch inference, one 16-row tile per warp at a time
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ W, const float* __restrict__ X,
                                                     int n, float* __restrict__ Y)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int warp = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * (blockDim.x / 32);
    for (int row0 = warp * 16; row0 < n; row0 += nwarps * 16)
    {
        auto x = [&](int r, int k) { return row0 + r < n ? X[(size_t)(row0 + r) * MLP_IN + k] : 0.f; };
        const float2 y = mlp_tile_forward_regs(W, x);
        if (t == 0)
        {
            if (row0 + g < n) Y[row0 + g] = y.x;
            if (row0 + g + 8 < n) Y[row0 + g + 8] = y.y;
        }
    }
}

// gradient of L = 0.5/n sum (y - t)^2 into G (zeroed by the caller), L into loss
__global__ void __launch_bounds__(128) k_mlp_grad(const float* __restrict__ W, const float* __restrict__ X,
                                                  const float* __restrict__ T, int n, float* G, float* loss)
{
    extern __shared__ unsigned char smem_raw[];
    WarpTile& s = reinterpret_cast<WarpTile*>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * (blockDim.x / 32);
    for (int row0 = warp * 16; row0 < n; row0 += nwarps * 16)
    {
        stage_tile(s, X, T, row0, n);
        tile_forward_smem(W, s);
        if (lane < 16 && row0 + lane < n)
        {
            const float d = s.y[lane] - s.T[lane];
            atomicAdd(loss, 0.5f * d * d / n);
        }
        tile_backward(W, s, min(16, n - row0), (float)n, G);
    }
}

// Mini-batch Adam (beta 0.9 / 0.999, eps 1e-8) over `epochs` passes of the data
// set, batches of 64 rows in a seeded order that changes every epoch; one block,
// 4 warps each taking one 16-row tile of the batch.  loss_out[e] = mean loss of
// epoch e as seen during the epoch.
__global__ void __launch_bounds__(128) k_mlp_train(float* W, float* m1, float* m2, float* G,
                                                   const float* __restrict__ X, const float* __restrict__ T,
                                                   int n, int epochs, float lr, unsigned seed, float* loss_out)
{
    extern __shared__ unsigned char smem_raw[];
    WarpTile& s = reinterpret_cast<WarpTile*>(smem_raw)[threadIdx.x >> 5];
    __shared__ float sh_loss;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int MB = 16 * MLP_WARPS;
    const int nbatch = (n + MB - 1) / MB;
    int step = 0;
    for (int ep = 0; ep < epochs; ++ep)
    {
        if (threadIdx.x == 0) sh_loss = 0.f;
        // batch order of this epoch: b = (a * i + c) mod nbatch with a coprime to nbatch
        unsigned a = (2654435761u * (seed + 1u) + 2u * (unsigned)ep) | 1u;
        for (int guard = 0; guard < 64; ++guard)
        {
            unsigned x = a, y = (unsigned)nbatch;
            while (y) { unsigned r = x % y; x = y; y = r; }
            if (x == 1u) break;
            a += 2u;
        }
        const unsigned c = seed * 40503u + (unsigned)ep * 9973u;
        for (int bi = 0; bi < nbatch; ++bi)
        {
            const int b = (int)(((unsigned long long)a * (unsigned)bi + c) % (unsigned)nbatch);
            const int row0 = b * MB, rows = min(MB, n - row0);
            for (int e = threadIdx.x; e < MLP_NPARAM; e += blockDim.x) G[e] = 0.f;
            __syncthreads();
            const int t0 = 16 * wid;
            if (t0 < rows)
            {
                stage_tile(s, X + (size_t)row0 * MLP_IN, T + row0, t0, rows);
                tile_forward_smem(W, s);
                if (lane < 16 && t0 + lane < rows)
                {
                    const float d = s.y[lane] - s.T[lane];
                    atomicAdd(&sh_loss, 0.5f * d * d / n);
                }
                tile_backward(W, s, min(16, rows - t0), (float)rows, G);
            }
            __syncthreads();
            ++step;
            const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
            const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
            for (int e = threadIdx.x; e < MLP_NPARAM; e += blockDim.x)
            {
                const float gr = G[e];
                m1[e] = b1 * m1[e] + (1.f - b1) * gr;
                m2[e] = b2 * m2[e] + (1.f - b2) * gr * gr;
                W[e] -= lr * (m1[e] / c1) / (sqrtf(m2[e] / c2) + eps);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0 && loss_out) loss_out[ep] = sh_loss;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
static size_t mlp_tile_smem() { return MLP_WARPS * sizeof(WarpTile); }

void launch_mlp_forward(const float* W, const float* X, int n, float* Y, cudaStream_t st)
{
    const int blocks = std::max(1, std::min((n + 16 * MLP_WARPS - 1) / (16 * MLP_WARPS), 148 * 8));
    k_mlp_forward<<<blocks, 32 * MLP_WARPS, 0, st>>>(W, X, n, Y);
}

void launch_mlp_grad(const float* W, const float* X, const float* T, int n, float* G, float* loss, cudaStream_t st)
{
    const size_t sm = mlp_tile_smem();
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const int blocks = std::max(1, std::min((n + 16 * MLP_WARPS - 1) / (16 * MLP_WARPS), 148 * 2));
    k_mlp_grad<<<blocks, 32 * MLP_WARPS, sm, st>>>(W, X, T, n, G, loss);
}

void launch_mlp_train(float* W, float* m1, float* m2, float* G, const float* X, const float* T, int n, int epochs,
                      float lr, unsigned seed, float* loss_out, cudaStream_t st)
{
    const size_t sm = mlp_tile_smem();
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_mlp_train<<<1, 32 * MLP_WARPS, sm, st>>>(W, m1, m2, G, X, T, n, epochs, lr, seed, loss_out);
}


}   // namespace abm

// ---------------------------------------------------------------------------
// C ABI on host buffers (include/abm_capi.h).  Each call allocates its device
// buffers, runs on a stream of its own on the current device and waits for it.
// ---------------------------------------------------------------------------
#include <cstring>
#include <string>
#include <vector>
#include "../../include/abm_capi.h"

namespace {

thread_local std::string g_mlp_err;

struct DevBufs {
    std::vector<void*> ptrs;
    cudaStream_t st = nullptr;
    ~DevBufs()
    {
        if (st) cudaStreamSynchronize(st);
        for (void* p : ptrs) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }
    template <class T> T* alloc(size_t count)
    {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

int mlp_fail(int code, const std::string& msg)
{
    g_mlp_err = msg;
    return code;
}

#define MLP_CK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    return mlp_fail(ABM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

}   // namespace

extern "C" {

const char* abm_mlp_last_error(void) { return g_mlp_err.c_str(); }

int abm_mlp_forward(const float* w, const float* X, int n, float* Y)
{
    g_mlp_err.clear();
    if (!w || n < 0 || (n > 0 && (!X || !Y))) return mlp_fail(ABM_ERR_ARG, "bad arguments");
    if (n == 0) return ABM_OK;
    DevBufs b;
    MLP_CK(cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking));
    float *dw = b.alloc<float>(abm::MLP_NPARAM), *dx = b.alloc<float>((size_t)n * abm::MLP_IN), *dy = b.alloc<float>(n);
    if (!dw || !dx || !dy) return mlp_fail(ABM_ERR_CUDA, "cudaMalloc failed");
    MLP_CK(cudaMemcpyAsync(dw, w, abm::MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, b.st));
    MLP_CK(cudaMemcpyAsync(dx, X, (size_t)n * abm::MLP_IN * sizeof(float), cudaMemcpyHostToDevice, b.st));
    abm::launch_mlp_forward(dw, dx, n, dy, b.st);
    MLP_CK(cudaGetLastError());
    MLP_CK(cudaMemcpyAsync(Y, dy, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, b.st));
    MLP_CK(cudaStreamSynchronize(b.st));
    return ABM_OK;
}

int abm_mlp_grad(const float* w, const float* X, const float* T, int n, float* grad, float* loss)
{
    g_mlp_err.clear();
    if (!w || !grad || !loss || n <= 0 || !X || !T) return mlp_fail(ABM_ERR_ARG, "bad arguments");
    DevBufs b;
    MLP_CK(cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking));
    float *dw = b.alloc<float>(abm::MLP_NPARAM), *dx = b.alloc<float>((size_t)n * abm::MLP_IN);
    float *dt = b.alloc<float>(n), *dg = b.alloc<float>(abm::MLP_NPARAM), *dl = b.alloc<float>(1);
    if (!dw || !dx || !dt || !dg || !dl) return mlp_fail(ABM_ERR_CUDA, "cudaMalloc failed");
    MLP_CK(cudaMemcpyAsync(dw, w, abm::MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, b.st));
    MLP_CK(cudaMemcpyAsync(dx, X, (size_t)n * abm::MLP_IN * sizeof(float), cudaMemcpyHostToDevice, b.st));
    MLP_CK(cudaMemcpyAsync(dt, T, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, b.st));
    MLP_CK(cudaMemsetAsync(dg, 0, abm::MLP_NPARAM * sizeof(float), b.st));
    MLP_CK(cudaMemsetAsync(dl, 0, sizeof(float), b.st));
    abm::launch_mlp_grad(dw, dx, dt, n, dg, dl, b.st);
    MLP_CK(cudaGetLastError());
    MLP_CK(cudaMemcpyAsync(grad, dg, abm::MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, b.st));
    MLP_CK(cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, b.st));
    MLP_CK(cudaStreamSynchronize(b.st));
    return ABM_OK;
}

int abm_mlp_train(float* w, const float* X, const float* T, int n, int epochs, float lr, unsigned seed,
                  float* loss_per_epoch)
{
    g_mlp_err.clear();
    if (!w || n <= 0 || !X || !T || epochs < 0 || !(lr > 0)) return mlp_fail(ABM_ERR_ARG, "bad arguments");
    DevBufs b;
    MLP_CK(cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking));
    float *dw = b.alloc<float>(abm::MLP_NPARAM), *m1 = b.alloc<float>(abm::MLP_NPARAM);
    float *m2 = b.alloc<float>(abm::MLP_NPARAM), *dg = b.alloc<float>(abm::MLP_NPARAM);
    float *dx = b.alloc<float>((size_t)n * abm::MLP_IN), *dt = b.alloc<float>(n);
    float* dl = b.alloc<float>(std::max(epochs, 1));
    if (!dw || !m1 || !m2 || !dg || !dx || !dt || !dl) return mlp_fail(ABM_ERR_CUDA, "cudaMalloc failed");
    MLP_CK(cudaMemcpyAsync(dw, w, abm::MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, b.st));
    MLP_CK(cudaMemcpyAsync(dx, X, (size_t)n * abm::MLP_IN * sizeof(float), cudaMemcpyHostToDevice, b.st));
    MLP_CK(cudaMemcpyAsync(dt, T, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, b.st));
    MLP_CK(cudaMemsetAsync(m1, 0, abm::MLP_NPARAM * sizeof(float), b.st));
    MLP_CK(cudaMemsetAsync(m2, 0, abm::MLP_NPARAM * sizeof(float), b.st));
    MLP_CK(cudaMemsetAsync(dl, 0, std::max(epochs, 1) * sizeof(float), b.st));
    if (epochs > 0) abm::launch_mlp_train(dw, m1, m2, dg, dx, dt, n, epochs, lr, seed, dl, b.st);
    MLP_CK(cudaGetLastError());
    MLP_CK(cudaMemcpyAsync(w, dw, abm::MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, b.st));
    if (loss_per_epoch && epochs > 0)
        MLP_CK(cudaMemcpyAsync(loss_per_epoch, dl, epochs * sizeof(float), cudaMemcpyDeviceToHost, b.st));
    MLP_CK(cudaStreamSynchronize(b.st));
    return ABM_OK;
}

}   // extern "C"
