// kernels.h -- host-side launchers shared between the translation units of librhmc_b200.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

struct rhmc_ctx;

namespace rhmc {

void launch_geometry(rhmc_ctx *c, int *table, int *eta);
void launch_gauge_from_ref(rhmc_ctx *c, const double *ref);
void launch_gauge_to_ref(rhmc_ctx *c, double *ref);
void launch_algebra_from_ref(rhmc_ctx *c, double *A, const double *ref, int antiherm);
void launch_algebra_to_ref(rhmc_ctx *c, double *ref, const double *A, int antiherm);
void launch_spinor_to_internal(rhmc_ctx *c, int fmt, void *dst, const double *src, int n);
void launch_spinor_from_internal(rhmc_ctx *c, int fmt, double *dst, const void *src, int n);
cudaError_t launch_dslash_f64_range(rhmc_ctx *c, cudaStream_t s, int p_out, void *out, const void *in, int k_lo, int k_count);

// Largest number of right-hand sides one Dslash launch carries.
constexpr int DSLASH_MAX_NR = 8;

// out[r] = alpha*y[r] + beta*(2*D in[r]) / 2 onto parity p_out, r < n, spinors `stride`
// elements apart.  With partials != NULL (n <= DSLASH_MAX_NR) each block writes, per RHS,
// Re<y,out> and |out|^2 into partials[block][2n]; *nblocks receives the grid size.
cudaError_t launch_dslash(rhmc_ctx *c, int fmt, int p_out, void *out, const void *in, size_t stride, int n,
                          const void *y, double alpha, double beta, double *partials, int *nblocks);
int dslash_grid(rhmc_ctx *c);
bool fmt_is_f64(int fmt);

}  // namespace rhmc
