// noalloc.cu -- FP64 true residuals |b_r - (M^dag M + sigma_i) x_{r,i}| that allocate no device
// memory (rhmc_true_residuals_noalloc).
//
// Who needs it: a caller that checks its solutions at a point where it must not call
// cudaMalloc.  Host programs that hand all device memory to their own pool at start-up treat
// any later allocation as an error; long Markov chains that share a GPU under a fixed memory
// budget cannot risk an out-of-memory failure hours into a run; and code that keeps work in
// flight on other streams cannot accept the device-wide synchronisation cudaMalloc may
// imply.  rhmc_true_residuals takes its two intermediate spinors and its reduction partials
// from the context's grow-on-demand workspace, which calls cudaMalloc the first time (and
// whenever a larger size is needed); this variant takes them from one fixed array instead.
//
// The call is host-synchronous: it waits for the context's stream and copies the residuals
// into the caller's host array before it returns.
//
// Scratch: the file-scope device array g_noalloc_scratch below, RHMC_NOALLOC_SCRATCH_BYTES
// (about 6.3 MB), which every GPU that loads the library holds until the process exits.
// Limits: at most RHMC_NOALLOC_MAX_VH sites per parity (e.g. 16^3 x 32) and at most
// RHMC_NOALLOC_MAX_SYSTEMS (rhs, shift) pairs per call; larger requests are rejected.
//
// The array is shared by every call on a device and keeps whatever the last call left in it.
// Each call writes every scratch word before reading it (the partials of one system are
// overwritten by the next, each result slot is written once), so nothing has to start at
// zero.  Two calls whose GPU work overlaps -- on different streams, or from different host
// threads -- use the same words and race; serialise them.
//
// Device address: host code cannot use the array's name as a device pointer (it names a host
// shadow).  The first call on a device, with that device current, looks the address up with
// cudaGetSymbolAddress and caches it (this set-up is part of that first call); make that first
// call before any stream capture.
#include <cmath>
#include <mutex>

#include "capi_util.h"
#include "context.h"
#include "kernels.h"

namespace rhmc {

constexpr int NA_BLOCK = 256;
constexpr int NA_MAX_GRID = (RHMC_NOALLOC_MAX_VH + NA_BLOCK - 1) / NA_BLOCK;
constexpr size_t NA_VEC = 3 * (size_t)RHMC_NOALLOC_MAX_VH;  // double2 elements per spinor
// layout: h spinor | t spinor | partials[NA_MAX_GRID] | results[RHMC_NOALLOC_MAX_SYSTEMS]
constexpr size_t NA_OFF_T = NA_VEC * sizeof(double2);
constexpr size_t NA_OFF_PART = 2 * NA_VEC * sizeof(double2);
constexpr size_t NA_OFF_RES = NA_OFF_PART + NA_MAX_GRID * sizeof(double);
static_assert(NA_OFF_RES + RHMC_NOALLOC_MAX_SYSTEMS * sizeof(double) <= RHMC_NOALLOC_SCRATCH_BYTES,
              "scratch layout exceeds the stated size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[RHMC_NOALLOC_SCRATCH_BYTES];

// per-block partial sums of |b - coef x - t|^2 for one system
__global__ void __launch_bounds__(NA_BLOCK) noalloc_resid_kernel(int Vh, double coef, const double2 *__restrict__ b,
                                                                  const double2 *__restrict__ x,
                                                                  const double2 *__restrict__ t, double *partials)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (k < Vh) {
        for (int c = 0; c < 3; c++) {
            const size_t o = (size_t)c * Vh + k;
            const double2 bv = b[o], xv = x[o], tv = t[o];
            const double re = bv.x - coef * xv.x - tv.x, im = bv.y - coef * xv.y - tv.y;
            v[0] += re * re + im * im;
        }
    }
    __shared__ double smem[32];
    block_sum<1>(v, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// one block: results[slot] = sum of partials[0..n) in block order
__global__ void __launch_bounds__(NA_BLOCK) noalloc_final_kernel(int n, const double *partials, double *results, int slot)
{
    double v[1] = {0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) v[0] += partials[i];
    __shared__ double smem[32];
    block_sum<1>(v, smem);
    if (threadIdx.x == 0) results[slot] = v[0];
}

static std::mutex g_na_mu;
static void *g_na_ptr[256];

// device address of the scratch array on `dev` (which must be current); looked up once
static int noalloc_scratch(int dev, unsigned char **out)
{
    if (dev < 0 || dev >= 256) return fail(RHMC_ERR_ARG, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_na_ptr[dev] = p;
    }
    *out = (unsigned char *)g_na_ptr[dev];
    return RHMC_OK;
}

}  // namespace rhmc

using namespace rhmc;

extern "C" int rhmc_true_residuals_noalloc(rhmc_ctx *c, int nshift, const double *shifts, int nrhs, const double *x,
                                           const double *b, double *out)
{
    if (!c || !shifts || !x || !b || !out || nshift < 1 || nrhs < 1) return fail(RHMC_ERR_ARG, "bad argument");
    if (c->Vh > RHMC_NOALLOC_MAX_VH)
        return fail(RHMC_ERR_ARG, "rhmc_true_residuals_noalloc: %ld sites per parity exceed the fixed scratch limit of %d",
                    c->Vh, RHMC_NOALLOC_MAX_VH);
    if ((long)nshift * nrhs > RHMC_NOALLOC_MAX_SYSTEMS)
        return fail(RHMC_ERR_ARG, "rhmc_true_residuals_noalloc: %ld systems exceed the limit of %d", (long)nshift * nrhs,
                    RHMC_NOALLOC_MAX_SYSTEMS);
    CK(cudaSetDevice(c->device));
    unsigned char *base = nullptr;
    int rc = noalloc_scratch(c->device, &base);
    if (rc) return rc;
    double2 *h = (double2 *)base, *t = (double2 *)(base + NA_OFF_T);
    double *part = (double *)(base + NA_OFF_PART), *res = (double *)(base + NA_OFF_RES);
    const int Vh = (int)c->Vh;
    const size_t stride = 3 * (size_t)Vh;
    const int grid = grid_for(Vh, NA_BLOCK);
    const double2 *xs = (const double2 *)x, *bs = (const double2 *)b;
    const int nsys = nshift * nrhs;
    for (int q = 0; q < nsys; q++) {
        const double2 *xq = xs + (size_t)q * stride;
        // t = -Deo Doe x with FP64 links (no derived copy, hence no allocation)
        cudaError_t e = launch_dslash(c, RHMC_LINKS_F64_18, 1, h, xq, stride, 1, nullptr, 0.0, 0.5, nullptr, nullptr);
        if (e == cudaSuccess) e = launch_dslash(c, RHMC_LINKS_F64_18, 0, t, h, stride, 1, nullptr, 0.0, -0.5, nullptr, nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "rhmc_true_residuals_noalloc");
        noalloc_resid_kernel<<<grid, NA_BLOCK, 0, c->stream>>>(Vh, c->mass * c->mass + shifts[q % nshift],
                                                               bs + (size_t)(q / nshift) * stride, xq, t, part);
        noalloc_final_kernel<<<1, NA_BLOCK, 0, c->stream>>>(grid, part, res, q);
        c->launches += 2;
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(out, res, (size_t)nsys * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int q = 0; q < nsys; q++) out[q] = std::sqrt(out[q]);
    return RHMC_OK;
}
