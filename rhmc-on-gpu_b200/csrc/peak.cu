// peak.cu -- CUDA-core FMA throughput microbenchmark (FP64 or FP32): the compute roofline of
// the FP64 force and link-exponentiation kernels, which are not tensor-core contractions.
//
// Method: every thread runs 8 independent FMA chains x <- x * a + b (a slightly below 1, so the
// values stay normal and finite) for `iters` rounds; 8 chains hide the FMA latency with a few
// warps per scheduler.  The grid is 8 blocks of 256 threads per SM.  One warm-up launch, then
// one timed launch with CUDA events on the context stream; flops = 2 * 8 * iters per thread.
#include "capi_util.h"
#include "context.h"

namespace rhmc {

template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T *out, int iters, T a, T b)
{
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = (T)(threadIdx.x + k) * (T)1e-3;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == (T)-1) out[blockIdx.x] = s;  // never true; keeps the chains live
}

static int fma_peak(rhmc_ctx *c, int fp64, double *tflops)
{
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    const int blocks = 8 * sms, threads = 256, iters = 1 << 14;
    void *out;
    CK(c->ws.get("fma_out", (size_t)blocks * sizeof(double), &out));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float ms = 0;
    for (int rep = 0; rep < 2; rep++) {
        CK(cudaEventRecord(e0, c->stream));
        if (fp64)
            fma_chain_kernel<double><<<blocks, threads, 0, c->stream>>>((double *)out, iters, 0.9999999, 1e-7);
        else
            fma_chain_kernel<float><<<blocks, threads, 0, c->stream>>>((float *)out, iters, 0.9999f, 1e-4f);
        CK(cudaEventRecord(e1, c->stream));
        c->launches++;
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(&ms, e0, e1));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaGetLastError());
    *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12;
    return RHMC_OK;
}

}  // namespace rhmc

extern "C" int rhmc_fma_peak(rhmc_ctx *c, int fp64, double *tflops)
{
    if (!c || !tflops) return rhmc::fail(RHMC_ERR_ARG, "null argument");
    return rhmc::fma_peak(c, fp64, tflops);
}
