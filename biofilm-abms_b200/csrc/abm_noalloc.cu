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
// zero: every slot a call reads is written earlier in the same call.
#include <cmath>
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

__global__ void k_na_setup(Ctrl* ctrl, int n, int n_dir)
{
    ctrl->n = n;
    ctrl->n_dir = n_dir;
    ctrl->status = 0;
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

thread_local char g_err[256];

}   // namespace

extern "C" const char* abm_noalloc_last_error(void) { return g_err; }

extern "C" int abm_cell_cell_forces_noalloc(const abm_params* p, const double* d_cells, int n, int ncols, int ld,
                                            const int* d_row_ptr, const int* d_col, int n_entries,
                                            const double* jkr_delta, const double* jkr_radius, int jkr_n,
                                            double* d_dEdq, void* stream)
{
    auto fail = [](int code, const char* msg) { strncpy(g_err, msg, sizeof(g_err) - 1); return code; };
    g_err[0] = 0;
    if (!p || (n > 0 && (!d_cells || !d_row_ptr || !d_dEdq)) || n < 0 || ld < n || n_entries < 0)
        return fail(ABM_ERR_ARG, "bad arguments");
    if (n > NA_MAX_CELLS) return fail(ABM_ERR_CAPACITY, "more than ABM_NOALLOC_MAX_CELLS cells");
    if (n_entries > NA_MAX_ENTRIES) return fail(ABM_ERR_CAPACITY, "more than ABM_NOALLOC_MAX_ENTRIES CSR entries");
    if (ncols < 21 || (p->adhesion_mode != 0 && ncols < 22))
        return fail(ABM_ERR_ARG, "cell arrays need 21 columns (22 with adhesion)");
    if (p->adhesion_mode != 0 && (!jkr_delta || !jkr_radius || jkr_n < 2 || jkr_n > NA_MAX_JKR))
        return fail(ABM_ERR_ARG, "adhesion needs a JKR table of 2..512 entries");
    if (p->pair_lanes != 4 && p->pair_lanes != 8 && p->pair_lanes != 16 && p->pair_lanes != 32)
        return fail(ABM_ERR_ARG, "pair_lanes must be 4, 8, 16 or 32");
    unsigned char* base = nullptr;
    const char* why = "";
    int rc = scratch_address(&base, &why);
    if (rc) return fail(rc, why);
    cudaStream_t st = (cudaStream_t)stream;
    Ctrl* ctrl = reinterpret_cast<Ctrl*>(base + OFF_CTRL);
    Geom* geom = reinterpret_cast<Geom*>(base + OFF_GEOM);
    Gen6* fcc = reinterpret_cast<Gen6*>(base + OFF_FCC);
    int* lower_end = reinterpret_cast<int*>(base + OFF_LOWER);
    int* rev = reinterpret_cast<int*>(base + OFF_REV);
    double4* jbuf = reinterpret_cast<double4*>(base + OFF_JBUF);
    double* tab = reinterpret_cast<double*>(base + OFF_JKR);

    ForceParams fp;
    fp.R = p->R; fp.Rcell = p->Rcell; fp.E0 = p->E0;
    fp.pf0 = (4. / 3.) * p->E0 * std::sqrt(p->R / 2);
    fp.pf1 = (4. / 3.) * p->Ecell * std::sqrt(p->Rcell / 2);
    fp.pf2 = (4. / 3.) * p->E0 * std::sqrt(p->R / 2) * std::pow(2 * (p->R - p->Rcell), 1.5);
    fp.max_overlap = 2 * (p->R - p->Rcell);
    fp.adhesion = p->adhesion_mode != 0;
    fp.stats = 0;
    fp.jkr_n = fp.adhesion ? jkr_n : 0;
    fp.jkr_step = fp.adhesion ? (jkr_delta[jkr_n - 1] - jkr_delta[0]) / double(jkr_n - 1) : 1.0;
    if (fp.adhesion)
    {
        // host -> device copies into the array; no allocation
        if (cudaMemcpyAsync(tab, jkr_delta, jkr_n * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(tab + NA_MAX_JKR, jkr_radius, jkr_n * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
            return fail(ABM_ERR_CUDA, "copy of the JKR table failed");
    }
    k_na_setup<<<1, 1, 0, st>>>(ctrl, n, n_entries);
    if (n > 0)
    {
        k_na_geom<<<(n + 255) / 256, 256, 0, st>>>(d_cells, n, ld, fp.adhesion, geom);
        launch_csr_rev(ctrl, d_row_ptr, d_col, lower_end, rev, n, st);
        launch_pair_force(geom, d_row_ptr, lower_end, d_col, rev, ctrl, fp, tab, tab + NA_MAX_JKR, fcc, jbuf,
                          p->pair_lanes, p->precision == ABM_PRECISION_MIXED, n, st, 1);
        launch_gen6_to_colmajor(fcc, n, d_dEdq, st);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ABM_ERR_CUDA, cudaGetErrorString(e));
    return ABM_OK;
}
