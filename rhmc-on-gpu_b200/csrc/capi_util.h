// capi_util.h -- error helpers for the extern "C" entry points.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

struct rhmc_ctx;

namespace rhmc {
int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
int stage_in(rhmc_ctx *c, const char *slot, const void *src, size_t bytes, int location, const void **dev);
}  // namespace rhmc

// return RHMC_ERR_CUDA from the enclosing entry point when a CUDA call fails
#define CK(call)                                                   \
    do {                                                           \
        cudaError_t ck_e_ = (call);                                \
        if (ck_e_ != cudaSuccess) return rhmc::cuda_fail(ck_e_, #call); \
    } while (0)
