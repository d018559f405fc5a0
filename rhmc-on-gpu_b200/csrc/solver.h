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
    void *x;              // FP64 internal spinors, [nrhs][nshift]
    int fresh = 1;        // 1: start from x = 0; 0: resume the state an FP64 phase left (FP32 links only)
    double tau = 0.0;     // > 0: stop each RHS once |r| <= tau |b| (to be resumed in lower precision);
                          // < 0: once |r| <= max(1e-4 |b|, min(-tau |b|, 1e7 res)) (FinInit)
    int ru_every = 0;     // > 0: reliable update of the base system every ru_every windows
};

struct MSolveInfo {
    int status;
    long graph_replays;
    int iters[8];
    double lambda[8];
    double b2[8];
    int ru_count;
};

// Replays `exec` on stream s until the device word *stop is non-zero (read one replay behind
// through a pinned host word, so the GPU never idles on the poll) or max_rep replays.
// *replays receives the number of replays issued.  Every CUDA call is checked: a failure
// returns RHMC_ERR_CUDA with the stream synchronised, and a loop that ends before the flag is
// seen leaves *stop_seen = 0.
int replay_until_stop(rhmc_ctx *c, cudaGraphExec_t exec, cudaStream_t s, const int *stop, long max_rep, long *replays,
                      int *stop_seen, const char *what);

// Multi-shift CG with links of format `fmt`; vectors in that format's precision.
int msolve_shifted(rhmc_ctx *c, int fmt, const MSolveArgs &A, MSolveInfo *info);

// |b_r - (M^dag M + sigma_{r,i}) x_{r,i}|^2 for every (r, i) in FP64 (links FP64/18).
// shifts: [nrhs][nshift]; x: FP64 internal [nrhs][nshift]; b: FP64 internal [nrhs]; out: [nrhs][nshift].
int true_residuals(rhmc_ctx *c, int nshift, const double *shifts, int nrhs, const double2 *x, const double2 *b, double *out);

}  // namespace rhmc
