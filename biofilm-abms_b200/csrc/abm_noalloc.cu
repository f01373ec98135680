// Cell-cell forces without any device allocation.
//
// Some callers cannot call cudaMalloc: their device memory belongs to another
// allocator (a framework's caching pool, or a fixed budget handed out up front),
// or they cannot accept the device-wide synchronisation that cudaMalloc/cudaFree
// bring into a step loop.  abm_cell_cell_forces_noalloc serves them: it runs the
// same two-pass pair-force kernels as abm_cell_cell_forces, on device buffers the
// caller already owns, and keeps all its scratch (cell records, reverse slots,
// the partner shares, a control block and the JKR table) in one file-scope
// __device__ array of fixed size.  That array exists on every GPU that loads
// this library, for the life of the process.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress (the array's name is only a
// host-side stand-in in host code) and caches it per device; make that first
// call before any stream capture.  Every call shares the one array, so calls
// whose work overlaps on the GPU (different streams, or different host threads
// on one device) race; serialise them.  Nothing in the array has to start at
// zero: every slot a call reads is written earlier in the same call (the control
// block by k_na_setup, the JKR table from the launch parameters, the records,
// reverse slots and shares by the kernels that read them later).
//
// The caller's neighbor CSR is checked on the device before any kernel indexes
// with it (k_na_check): row bounds inside [0, n_entries] and non-decreasing,
// row_ptr[0] = 0 and row_ptr[n] = n_entries, every column in [0, n) and not the row
// itself, rows strictly ascending, and each entry (i, j) matched by an entry (j, i).
// A CSR that fails leaves the pair kernels with no cells to process, fills d_dEdq
// with NaN and is reported by abm_cell_cell_forces_noalloc_status.  The pair
// kernels write the partner share jbuf[rev[k]] at the slot the reverse search
// found, which the check guarantees lies inside [0, n_entries).
#include <cmath>
#include <cstddef>
#include <cstring>
#include <mutex>
#include "abm_kernels.cuh"
#include "../../include/abm_capi.h"

using namespace abm;

namespace {

// Limits of one call (also in include/abm_capi.h)
const int NA_MAX_CELLS = ABM_NOALLOC_MAX_CELLS;        // 32768
const int NA_MAX_ENTRIES = ABM_NOALLOC_MAX_ENTRIES;    // 524288 directed CSR entries
const int NA_MAX_JKR = 512;

// status bits of a rejected CSR (the control block's status word)
const int NA_BAD_BOUNDS = 1 << 8;    // row_ptr out of [0, n_entries], decreasing, or ends not 0 / n_entries
const int NA_BAD_COLUMN = 1 << 9;    // a column outside [0, n) or equal to its row
const int NA_BAD_ORDER = 1 << 10;    // a row not strictly ascending
const int NA_BAD_SYMMETRY = 1 << 11; // an entry (i, j) without its entry (j, i)
const int NA_BAD = NA_BAD_BOUNDS | NA_BAD_COLUMN | NA_BAD_ORDER | NA_BAD_SYMMETRY;

// byte offsets inside the scratch array, each 256-byte aligned
const size_t OFF_CTRL = 0;
const size_t OFF_GEOM = (sizeof(Ctrl) + 255) / 256 * 256;
const size_t OFF_FCC = OFF_GEOM + (size_t)NA_MAX_CELLS * sizeof(Geom);
const size_t OFF_LOWER = OFF_FCC + (size_t)NA_MAX_CELLS * sizeof(Gen6);
const size_t OFF_REV = OFF_LOWER + (size_t)NA_MAX_CELLS * sizeof(int);
const size_t OFF_JBUF = OFF_REV + (size_t)NA_MAX_ENTRIES * sizeof(int);
const size_t OFF_JKR = OFF_JBUF + (size_t)NA_MAX_ENTRIES * sizeof(double4);
const size_t SCRATCH_BYTES = OFF_JKR + 2 * (size_t)NA_MAX_JKR * sizeof(double);

static_assert(OFF_FCC % 256 == 0 && OFF_LOWER % 256 == 0 && OFF_REV % 256 == 0 &&
              OFF_JBUF % 256 == 0 && OFF_JKR % 256 == 0, "scratch regions must stay 256-byte aligned");

// The JKR table travels as a launch parameter (8 KB), so a call reads the caller's
// host arrays only while it runs and needs no host-to-device copy.
struct JkrParam {
    int n;
    double delta[NA_MAX_JKR];
    double radius[NA_MAX_JKR];
};

}   // namespace

// The scratch array (about 21 MB).  Host code must not pass this name to a kernel:
// on the host it is only a stand-in; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_abm_noalloc_scratch[SCRATCH_BYTES];

namespace {

std::mutex g_mu;
void* g_scratch_addr[64];
bool g_scratch_ready[64];

// once per device, with that device current
int scratch_address(unsigned char** out, const char** why)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { *why = "no current CUDA device"; return ABM_ERR_CUDA; }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ready[dev])
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_abm_noalloc_scratch);
        if (e != cudaSuccess || !p) { *why = "cudaGetSymbolAddress failed"; return ABM_ERR_CUDA; }
        g_scratch_addr[dev] = p;
        g_scratch_ready[dev] = true;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
    return ABM_OK;
}

// Every control-block field the pair kernels read, before anything else runs.  The
// cell count stays 0 until the CSR has passed its check (k_na_commit).
__global__ void k_na_setup(Ctrl* ctrl, int n_entries, const __grid_constant__ JkrParam jkr, double* tab)
{
    if (threadIdx.x == 0)
    {
        ctrl->n = 0;
        ctrl->n_dir = n_entries;
        ctrl->status = 0;
        ctrl->halted = 0;
        ctrl->iter = 0;
        ctrl->st_ovl_bits[0] = 0ull;
        ctrl->st_ovl_bits[1] = 0ull;
    }
    for (int k = threadIdx.x; k < jkr.n; k += blockDim.x)
    {
        tab[k] = jkr.delta[k];
        tab[NA_MAX_JKR + k] = jkr.radius[k];
    }
}

// The caller's CSR, one warp per row.  Every index read stays inside row_ptr[0..n]
// and col[0..n_entries): a partner row's bounds are checked before they are used,
// and the reverse search runs only inside a row whose bounds passed.
__global__ void __launch_bounds__(256) k_na_check(const int* __restrict__ row_ptr, const int* __restrict__ col,
                                                  int n, int n_entries, Ctrl* ctrl)
{
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x / 32);
    int bad = 0;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps)
    {
        const int r0 = row_ptr[i], r1 = row_ptr[i + 1];
        if (r0 < 0 || r1 < r0 || r1 > n_entries || (i == 0 && r0 != 0) || (i == n - 1 && r1 != n_entries))
        {
            bad |= NA_BAD_BOUNDS;
            continue;
        }
        for (int k = r0 + lane; k < r1; k += 32)
        {
            const int j = col[k];
            if (j < 0 || j >= n || j == i) { bad |= NA_BAD_COLUMN; continue; }
            if (k > r0 && !(col[k - 1] < j)) bad |= NA_BAD_ORDER;
            const int a0 = row_ptr[j], b0 = row_ptr[j + 1];
            if (a0 < 0 || b0 < a0 || b0 > n_entries) { bad |= NA_BAD_BOUNDS; continue; }
            int a = a0, b = b0;
            while (a < b) { const int mid = (a + b) >> 1; if (col[mid] < i) a = mid + 1; else b = mid; }
            if (a >= b0 || col[a] != i) bad |= NA_BAD_SYMMETRY;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    if (lane == 0 && bad) atomicOr(&ctrl->status, bad);
}

__global__ void k_na_commit(Ctrl* ctrl, int n)
{
    ctrl->n = (ctrl->status & NA_BAD) ? 0 : n;
}

// column-major cells (indices.hpp order, gamma in column 21 when present) -> records
__global__ void k_na_geom(const double* __restrict__ cm, int n, int ld, int has_gamma, Geom* geom)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Geom g;
    g.rx = cm[(size_t)1 * ld + i]; g.ry = cm[(size_t)2 * ld + i]; g.rz = cm[(size_t)3 * ld + i];
    g.h = cm[(size_t)14 * ld + i];
    g.nx = cm[(size_t)4 * ld + i]; g.ny = cm[(size_t)5 * ld + i]; g.nz = cm[(size_t)6 * ld + i];
    g.gamma = has_gamma ? cm[(size_t)21 * ld + i] : 0.0;
    geom[i] = g;
}

// dE/dq records -> the caller's n x 6 column-major output; NaN everywhere when the
// CSR was rejected (the pair kernels did not run)
__global__ void k_na_out(const Gen6* __restrict__ g, const Ctrl* ctrl, int n, double* cm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool rejected = (ctrl->status & NA_BAD) != 0;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    const Gen6 v = g[i];
    for (int k = 0; k < 6; ++k) cm[(size_t)k * n + i] = rejected ? nan : v.f[k];
}

thread_local char g_err[256];

int na_fail(int code, const char* msg)
{
    strncpy(g_err, msg, sizeof(g_err) - 1);
    g_err[sizeof(g_err) - 1] = 0;
    return code;
}

}   // namespace

extern "C" const char* abm_noalloc_last_error(void) { return g_err; }

extern "C" int abm_cell_cell_forces_noalloc(const abm_params* p, const double* d_cells, int n, int ncols, int ld,
                                            const int* d_row_ptr, const int* d_col, int n_entries,
                                            const double* jkr_delta, const double* jkr_radius, int jkr_n,
                                            double* d_dEdq, void* stream)
{
    g_err[0] = 0;
    if (!p || n < 0 || ld < n || n_entries < 0 || (n > 0 && (!d_cells || !d_row_ptr || !d_dEdq)) ||
        (n_entries > 0 && !d_col))
        return na_fail(ABM_ERR_ARG, "bad arguments");
    if (n > NA_MAX_CELLS) return na_fail(ABM_ERR_CAPACITY, "more than ABM_NOALLOC_MAX_CELLS cells");
    if (n_entries > NA_MAX_ENTRIES) return na_fail(ABM_ERR_CAPACITY, "more than ABM_NOALLOC_MAX_ENTRIES CSR entries");
    if (n == 0 && n_entries != 0) return na_fail(ABM_ERR_ARG, "CSR entries without cells");
    if (p->dims == 2) return na_fail(ABM_ERR_ARG, "the no-alloc entry point serves the 3-D model only");
    if (p->dims != 0 && p->dims != 3) return na_fail(ABM_ERR_ARG, "dims must be 3 (or 0)");
    if (p->adhesion_mode != 0 && p->adhesion_mode != 1) return na_fail(ABM_ERR_ARG, "adhesion_mode must be 0 or 1");
    if (p->precision != ABM_PRECISION_FP64 && p->precision != ABM_PRECISION_MIXED)
        return na_fail(ABM_ERR_ARG, "precision must be ABM_PRECISION_FP64 or ABM_PRECISION_MIXED");
    if (ncols < 21 || (p->adhesion_mode != 0 && ncols < 22))
        return na_fail(ABM_ERR_ARG, "cell arrays need 21 columns (22 with adhesion)");
    if (p->adhesion_mode != 0)
    {
        if (!jkr_delta || !jkr_radius || jkr_n < 2 || jkr_n > NA_MAX_JKR)
            return na_fail(ABM_ERR_ARG, "adhesion needs a JKR table of 2..512 entries");
        for (int k = 1; k < jkr_n; ++k)
            if (!(jkr_delta[k] > jkr_delta[k - 1])) return na_fail(ABM_ERR_ARG, "JKR overlap mesh must be increasing");
    }
    if (p->pair_lanes != 4 && p->pair_lanes != 8 && p->pair_lanes != 16 && p->pair_lanes != 32)
        return na_fail(ABM_ERR_ARG, "pair_lanes must be 4, 8, 16 or 32");
    unsigned char* base = nullptr;
    const char* why = "";
    int rc = scratch_address(&base, &why);
    if (rc) return na_fail(rc, why);
    cudaStream_t st = (cudaStream_t)stream;
    Ctrl* ctrl = reinterpret_cast<Ctrl*>(base + OFF_CTRL);
    Geom* geom = reinterpret_cast<Geom*>(base + OFF_GEOM);
    Gen6* fcc = reinterpret_cast<Gen6*>(base + OFF_FCC);
    int* lower_end = reinterpret_cast<int*>(base + OFF_LOWER);
    int* rev = reinterpret_cast<int*>(base + OFF_REV);
    double4* jbuf = reinterpret_cast<double4*>(base + OFF_JBUF);
    double* tab = reinterpret_cast<double*>(base + OFF_JKR);

    ForceParams fp;
    memset(&fp, 0, sizeof(fp));
    fp.R = p->R; fp.Rcell = p->Rcell; fp.E0 = p->E0;
    fp.pf0 = (4. / 3.) * p->E0 * std::sqrt(p->R / 2);
    fp.pf1 = (4. / 3.) * p->Ecell * std::sqrt(p->Rcell / 2);
    fp.pf2 = (4. / 3.) * p->E0 * std::sqrt(p->R / 2) * std::pow(2 * (p->R - p->Rcell), 1.5);
    fp.max_overlap = 2 * (p->R - p->Rcell);
    fp.adhesion = p->adhesion_mode != 0;
    fp.stats = 0;
    fp.jkr_n = fp.adhesion ? jkr_n : 0;
    fp.jkr_step = fp.adhesion ? (jkr_delta[jkr_n - 1] - jkr_delta[0]) / double(jkr_n - 1) : 1.0;
    JkrParam jp;
    jp.n = fp.jkr_n;
    for (int k = 0; k < jp.n; ++k) { jp.delta[k] = jkr_delta[k]; jp.radius[k] = jkr_radius[k]; }

    k_na_setup<<<1, 128, 0, st>>>(ctrl, n_entries, jp, tab);
    if (n > 0)
    {
        k_na_check<<<(n + 7) / 8, 256, 0, st>>>(d_row_ptr, d_col, n, n_entries, ctrl);
        k_na_commit<<<1, 1, 0, st>>>(ctrl, n);
        k_na_geom<<<(n + 255) / 256, 256, 0, st>>>(d_cells, n, ld, fp.adhesion, geom);
        launch_csr_rev(ctrl, d_row_ptr, d_col, lower_end, rev, n, st);
        launch_pair_force(geom, d_row_ptr, lower_end, d_col, rev, ctrl, fp, tab, tab + NA_MAX_JKR, fcc, jbuf,
                          p->pair_lanes, p->precision == ABM_PRECISION_MIXED, n, st, 1);
        k_na_out<<<(n + 255) / 256, 256, 0, st>>>(fcc, ctrl, n, d_dEdq);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(ABM_ERR_CUDA, cudaGetErrorString(e));
    return ABM_OK;
}

extern "C" int abm_cell_cell_forces_noalloc_status(void* stream)
{
    g_err[0] = 0;
    unsigned char* base = nullptr;
    const char* why = "";
    int rc = scratch_address(&base, &why);
    if (rc) return na_fail(rc, why);
    cudaStream_t st = (cudaStream_t)stream;
    int status = 0;
    if (cudaMemcpyAsync(&status, base + OFF_CTRL + offsetof(Ctrl, status), sizeof(int), cudaMemcpyDeviceToHost, st)
            != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
        return na_fail(ABM_ERR_CUDA, "reading the status of the last call failed");
    if (!(status & NA_BAD)) return ABM_OK;
    char msg[200] = "the neighbor CSR of the last call was rejected:";
    if (status & NA_BAD_BOUNDS) strncat(msg, " row bounds", sizeof(msg) - strlen(msg) - 1);
    if (status & NA_BAD_COLUMN) strncat(msg, " column range", sizeof(msg) - strlen(msg) - 1);
    if (status & NA_BAD_ORDER) strncat(msg, " row order", sizeof(msg) - strlen(msg) - 1);
    if (status & NA_BAD_SYMMETRY) strncat(msg, " symmetry", sizeof(msg) - strlen(msg) - 1);
    return na_fail(ABM_ERR_ARG, msg);
}
