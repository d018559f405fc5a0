// solver.h -- internal interfaces of the multi-shift solvers.
#pragma once
#include <cuda_runtime.h>

struct rhmc_ctx;

namespace rhmc {

struct MSolveArgs {
    int nshift, nrhs;
    const double *shift;  // absolute shifts sigma_{r,i}, [nrhs][nshift] (each RHS its own pole set)
    const double *base;   // [nrhs]: the iterated operator of RHS r is M^dag M + base[r]
    const double *tgt;    // per-shift freezing thresholds on sqrt(delta zeta^2)
    double res_base;      // stop when sqrt(|r|^2) <= res_base
    int max_iter;
    int stop_on_frozen;
    int chunk;            // iterations per captured graph (the multi-shift loop uses its window, MS_WIN)
    const void *b;        // FP64 internal spinors, nrhs of them
    void *x;              // internal spinors of the link format's precision, [nrhs][nshift]
};

struct MSolveInfo {
    int status;
    long graph_replays;
    int iters[8];
    double lambda[8];
    double b2[8];
};

// Multi-shift CG with links of format `fmt`; vectors in that format's precision.
int msolve_shifted(rhmc_ctx *c, int fmt, const MSolveArgs &A, MSolveInfo *info);

// |b_r - (M^dag M + sigma_{r,i}) x_{r,i}|^2 for every (r, i) in FP64 (links FP64/18).
// shifts: [nrhs][nshift]; x: FP64 internal [nrhs][nshift]; b: FP64 internal [nrhs]; out: [nrhs][nshift].
int true_residuals(rhmc_ctx *c, int nshift, const double *shifts, int nrhs, const double2 *x, const double2 *b, double *out);

}  // namespace rhmc
