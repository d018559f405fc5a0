// msolve.cuh -- multi-shift conjugate gradient on (M^dag M + sigma_i) x_i = b over even sites.
//
// Algorithm: Jegerlehner's multi-shift CG (hep-lat/9612014) exactly as the reference's CPU
// solver runs it (multips_shifted_invert, lib/Action/Inverter/inverter.cc:142-299): x_i = 0,
// r = p = p_i = b; per iteration
//   s = (M^dag M + sigma_0) p, alpha = Re<p,s>, omega = -delta/alpha
//   zeta'''_i = zeta_i zeta''_i omega_prev / (omega gamma (zeta_i - zeta''_i)
//                                               + zeta_i omega_prev (1 - sigma_i omega))
//   omega_i = omega zeta'''_i / zeta''_i ;  x_i -= omega_i p_i
//   r += omega s, lambda = |r|^2, gamma = lambda/delta, p = r + gamma p
//   gamma_i = gamma zeta'''_i omega_i / (zeta''_i omega) ; p_i = zeta'''_i r + gamma_i p_i
//   freeze shift i when sqrt(delta zeta''_i^2) < tgt_i (lagged residual, as inverter.cc:275-279)
// stopping when sqrt(lambda) <= res (inverter.cc:287), when every shift is frozen (the GPU
// solver's criterion, cuda_inverter.cu:777-785) or at max_iter.  sigma_0 is the base shift
// (0 in the reference; the mixed solver uses the smallest pole) and sigma_i are relative to it.
//
// Kernel sequence per iteration (one CUDA graph replays a window of MS_WIN iterations):
//   K1 D_oe:    h = D_oe p                                   (Dslash, NR right-hand sides)
//   K2 D_eo:    s = (m^2+sigma_0) p - D_eo h, Re<p,s>        (Dslash epilogue + FP64 reduction;
//               the last block computes omega, zeta''', omega_i for every RHS)
//   K3 resid:   r += omega s, |r|^2 into the window's ring   (last block: gamma, gamma_i, freezing,
//               convergence, stop flag)
//   K4 update:  p = r + gamma p
// and once per window the flush kernel applies the window's x_i -= omega_i p_i and
// p_i = zeta''' r + gamma_i p_i of every shift, composed from the recorded scalars and residuals.
// Scalars live in device memory (MSState) and never leave the GPU during the solve; the host
// only polls the stop flag between graph replays.
#pragma once
#include "dslash.cuh"

namespace rhmc {

constexpr int MS_MAX_SHIFT = 32;
constexpr int MS_MAX_RHS = 8;
constexpr int MS_WIN = 8;  // iterations per delayed-update window (= iterations per graph replay)
constexpr int VEC_BLOCK = 256;

struct MSRhs {
    double delta, omega, omega_prev, gamma, lambda, alpha, b2;
    double res;        // this phase stops the RHS when sqrt(lambda) <= res
    int iter;          // iterations performed
    int running;       // this iteration updates the RHS
    int running_next;  // still running after this iteration
    int rslot;         // ring slot holding the current residual
    int i0;            // index of the base shift (relative shift 0) among this RHS's poles
    double ru_best;    // smallest true |r|^2 seen at a reliable update
    int ru_stall;      // reliable updates since ru_best last fell by 4x
    double zeta_i[MS_MAX_SHIFT], zeta_ii[MS_MAX_SHIFT], zeta_iii[MS_MAX_SHIFT];
    double omegas[MS_MAX_SHIFT], gammas[MS_MAX_SHIFT];
    int active[MS_MAX_SHIFT];       // shift updated in this iteration
    int active_next[MS_MAX_SHIFT];  // after the freezing test
    double shift[MS_MAX_SHIFT];     // sigma_{r,i} - sigma_{r,0}: this RHS's poles relative to its base
    // the scalars of each iteration m of the current window, for the delayed shifted updates:
    // x_i -= h_om p_i, then p_i = h_ze r_m + h_ga p_i, applied by ms_flush_kernel when h_act
    double h_om[MS_MAX_SHIFT][MS_WIN], h_ga[MS_MAX_SHIFT][MS_WIN], h_ze[MS_MAX_SHIFT][MS_WIN];
    int h_act[MS_MAX_SHIFT][MS_WIN];
};

struct MSState {
    int stop;     // every RHS finished: K1-K3 skip
    int stop_k4;  // set by the first skipped K1 so that K4 skips from the next iteration on
    int wpos;     // iterations done in the current window (the residual of iteration m is in ring slot m-1)
    int status;   // 0 ok, 1 iteration cap, 2 non-finite reduction
    int nshift, nrhs, max_iter;
    int stop_on_frozen;             // also stop when every shift is frozen
    double res;                     // base residual target: stop when sqrt(lambda) <= res
    double tau;                     // > 0: this phase stops an RHS once sqrt(lambda) <= tau |b| (a
                                    // later phase in lower precision resumes it)
    double tgt[MS_MAX_SHIFT];       // freezing threshold for sqrt(delta zeta''^2)
    // reliable updates (resumed lower-precision phase): every ru_every windows the base residual
    // is recomputed in FP64 from the FP64 base solution and the base direction re-synchronised
    int ru_every, ru_windows, ru_now, ru_count;
    MSRhs rhs[MS_MAX_RHS];
};

// ------------------------------------------------------------------ last-block scalar steps
// The FP32 part of the precision schedule, with its FP64 reliable updates, leaves the shifted
// systems near 1e-7 of the residual at which it took over (a 1e-10 |b| target is met with the
// hand-over at 1e-3 |b|): the automatic hand-over (tau < 0) is therefore placed at most this far
// above the final target, so that deep targets do not leave every system to the refinement.
constexpr double MS_TAU_REACH = 1e7;
// ... but not below 1e-4 |b|: targets at the FP64 rounding floor of the smallest poles leave
// those systems to the refinement whatever the hand-over, and an earlier one only lengthens the
// FP64 part
constexpr double MS_TAU_MIN = 1e-4;

struct FinInit {
    MSState *st;
    __device__ void operator()(const double *tot) const
    {
        if (threadIdx.x != 0) return;
        for (int r = 0; r < st->nrhs; r++) {
            MSRhs &q = st->rhs[r];
            q.b2 = tot[r];
            q.delta = tot[r];
            q.omega = 1.0;
            q.omega_prev = 1.0;
            q.gamma = 0.0;
            q.lambda = tot[r];
            q.alpha = 0.0;
            q.iter = 0;
            q.rslot = MS_WIN - 1;
            // precision schedule: the FP64 part ends at tau |b| (tau > 0), or with tau < 0 at
            // -tau |b| but no more than MS_TAU_REACH above the final target
            const double nb = sqrt(tot[r]);
            q.res = st->tau > 0.0   ? fmax(st->res, st->tau * nb)
                    : st->tau < 0.0 ? fmax(st->res, fmax(MS_TAU_MIN * nb, fmin(-st->tau * nb, MS_TAU_REACH * st->res)))
                                    : st->res;
            q.running = 1;
            q.running_next = (tot[r] > 0.0) ? 1 : 0;  // b == 0: x = 0 is exact
            if (!isfinite(tot[r])) {
                st->status = 2;
                q.running_next = 0;
            }
            for (int i = 0; i < st->nshift; i++) {
                q.zeta_i[i] = 1.0;
                q.zeta_ii[i] = 1.0;
                q.zeta_iii[i] = 1.0;
                q.omegas[i] = 0.0;
                q.gammas[i] = 0.0;
                q.active[i] = 1;
                q.active_next[i] = 1;
            }
        }
        st->stop = 0;
        st->stop_k4 = 0;
        int any = 0;
        for (int r = 0; r < st->nrhs; r++) any |= st->rhs[r].running_next;
        if (!any) st->stop = 1;
    }
};

// FinAlpha and FinLambda run in every thread of the reduction's last block: thread 0 steps the
// scalars of each right-hand side, then one thread per (rhs, shift) the shifted recurrences
// (independent divisions in parallel instead of one thread's serial chain).
template <int NR>
struct FinAlpha {
    MSState *st;
    __device__ void operator()(const double *tot) const
    {
        if (threadIdx.x == 0) {
            for (int r = 0; r < NR; r++) {
                MSRhs &q = st->rhs[r];
                q.running = q.running_next;
                if (!q.running) continue;
                q.alpha = tot[r];
                if (!isfinite(q.alpha) || q.alpha == 0.0) {
                    st->status = 2;
                    st->stop = 1;
                    q.running = 0;
                    q.running_next = 0;
                    continue;
                }
                q.omega_prev = q.omega;
                q.omega = -q.delta / q.alpha;
            }
        }
        __syncthreads();
        const int ns = st->nshift, wp = st->wpos;
        for (int t = threadIdx.x; t < NR * ns; t += blockDim.x) {
            const int r = t / ns, i = t % ns;
            MSRhs &q = st->rhs[r];
            const int act = q.running ? q.active_next[i] : 0;
            q.h_act[i][wp] = act;
            if (!q.running) continue;
            q.active[i] = act;
            if (!act) continue;
            const double zi = q.zeta_i[i], zii = q.zeta_ii[i];
            const double ziii = (zi * zii * q.omega_prev) /
                                (q.omega * q.gamma * (zi - zii) + zi * q.omega_prev * (1.0 - q.shift[i] * q.omega));
            q.zeta_iii[i] = ziii;
            q.omegas[i] = q.omega * ziii / zii;
            q.h_om[i][wp] = q.omegas[i];
        }
    }
};

template <int NR>
struct FinLambda {
    MSState *st;
    __device__ void operator()(const double *tot) const
    {
        if (threadIdx.x == 0) {
            for (int r = 0; r < NR; r++) {
                MSRhs &q = st->rhs[r];
                if (!q.running) continue;
                q.lambda = tot[r];
                q.rslot = st->wpos;
                if (!isfinite(q.lambda)) {
                    st->status = 2;
                    q.running_next = 0;
                    continue;
                }
                q.gamma = q.lambda / q.delta;
            }
        }
        __syncthreads();
        const int ns = st->nshift, wp = st->wpos;
        for (int t = threadIdx.x; t < NR * ns; t += blockDim.x) {
            const int r = t / ns, i = t % ns;
            MSRhs &q = st->rhs[r];
            if (!q.running || !isfinite(q.lambda) || !q.active[i]) continue;
            q.gammas[i] = q.gamma * q.zeta_iii[i] * q.omegas[i] / (q.zeta_ii[i] * q.omega);
            q.h_ga[i][wp] = q.gammas[i];
            q.h_ze[i][wp] = q.zeta_iii[i];
            const double fact = sqrt(q.delta * q.zeta_ii[i] * q.zeta_ii[i]);
            q.active_next[i] = (fact < st->tgt[i]) ? 0 : 1;
            q.zeta_i[i] = q.zeta_ii[i];
            q.zeta_ii[i] = q.zeta_iii[i];
        }
        __syncthreads();
        if (threadIdx.x != 0) return;
        int any = 0;
        for (int r = 0; r < NR; r++) {
            MSRhs &q = st->rhs[r];
            if (!q.running || !isfinite(q.lambda)) continue;
            int nact = 0;
            for (int i = 0; i < ns; i++) nact += q.active[i] ? q.active_next[i] : 0;
            q.delta = q.lambda;
            q.iter++;
            int done = (sqrt(q.lambda) <= q.res) || (st->stop_on_frozen && nact == 0);
            if (!done && q.iter >= st->max_iter) {
                done = 1;
                st->status = (st->status == 0) ? 1 : st->status;
            }
            q.running_next = !done;
            any |= q.running_next;
        }
        for (int r = NR; r < st->nrhs; r++) any |= st->rhs[r].running_next;
        if (!any) st->stop = 1;
        st->wpos++;
    }
};

// end of a window (after ms_flush_kernel has read its scalars)
struct FinWindow {
    MSState *st;
    __device__ void operator()(const double *) const
    {
        if (threadIdx.x == 0) st->wpos = 0;
    }
};

// ------------------------------------------------------------------ vector kernels
template <typename Rv>
struct MSVec {
    typedef typename SpinorT<Rv>::elem E;
};

// Layout of the base vectors (residual ring, p, h, s) of NR right-hand sides in precision Rv:
// FP32 packed P at a time (PackS; a 32-byte element holds 4 right-hand sides of one colour and
// site, 16 bytes 2 of them), so that the Dslash of the batch loads P right-hand sides per
// instruction; plane per RHS (P = 1) for FP64, whose 16-byte plane loads are already wide (its
// packed form, 2 per 32 bytes, was faster for 4 right-hand sides at 32^4 but slower for 2 and 8
// in trajectories), and for batch widths that do not split into packs.  The shifted solutions
// and directions, the right-hand sides b and every caller-visible vector keep the plane layout.
template <typename Rv, int NR>
struct BasePack {
    static constexpr int P = sizeof(Rv) == 4 ? (NR % 4 == 0 ? 4 : (NR % 2 == 0 ? 2 : 1)) : 1;
};

// index, in complex numbers, of RHS j, colour c, site k in a set of NR base vectors
template <typename Rv, int NR>
__host__ __device__ __forceinline__ size_t bidx(int j, int c, int k, int Vh)
{
    constexpr int P = BasePack<Rv, NR>::P;
    return ((size_t)((j / P) * 3 + c) * Vh + k) * P + (j % P);
}

// x_i = 0, r_0 = p = p_i = b (b FP64 internal), |b|^2.  r_0 goes to the last slot of the
// residual ring (the slot the first iteration reads).  Base vectors (ring, p) are stored in Rv,
// the shifted solutions and directions (x, ps) in Rx.
template <typename Rv, typename Rx, int NR>
__global__ void __launch_bounds__(VEC_BLOCK) ms_init_kernel(int Vh, int nshift, size_t stride, const double2 *__restrict__ b,
                                                             typename MSVec<Rv>::E *ring, typename MSVec<Rv>::E *p,
                                                             typename MSVec<Rx>::E *ps, typename MSVec<Rx>::E *x,
                                                             double *partials, unsigned *ticket, MSState *st)
{
    typename MSVec<Rv>::E *r = ring + (size_t)(MS_WIN - 1) * NR * stride;
    typedef typename MSVec<Rv>::E E;
    typedef typename MSVec<Rx>::E EX;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double red[NR];
#pragma unroll
    for (int j = 0; j < NR; j++) red[j] = 0.0;
    if (k < Vh) {
#pragma unroll
        for (int j = 0; j < NR; j++) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const size_t o = j * stride + (size_t)c * Vh + k, ob = bidx<Rv, NR>(j, c, k, Vh);
                const double2 v = b[o];
                red[j] += dot2(v.x, v.x, v.y, v.y);
                E e;
                e.x = (Rv)v.x;
                e.y = (Rv)v.y;
                r[ob] = e;
                p[ob] = e;
                EX ex, z;
                ex.x = (Rx)v.x;
                ex.y = (Rx)v.y;
                z.x = 0;
                z.y = 0;
                for (int i = 0; i < nshift; i++) {
                    const size_t oi = (size_t)(j * nshift + i) * stride + (size_t)c * Vh + k;
                    ps[oi] = ex;
                    x[oi] = z;
                }
            }
        }
    }
    FinInit fin{st};
    reduce_finalize<NR>(red, partials, ticket, fin);
}

// r_m = r_{m-1} + omega s (ring slots wpos-1 -> wpos), |r_m|^2 per RHS
template <typename Rv, int NR>
__global__ void __launch_bounds__(VEC_BLOCK) ms_resid_kernel(int Vh, size_t stride, typename MSVec<Rv>::E *ring,
                                                              const typename MSVec<Rv>::E *__restrict__ s, double *partials,
                                                              unsigned *ticket, MSState *st)
{
    typedef typename MSVec<Rv>::E E;
    if (*(volatile int *)&st->stop) return;
    const int wp = *(volatile const int *)&st->wpos;
    const E *rprev = ring + (size_t)((wp + MS_WIN - 1) % MS_WIN) * NR * stride;
    E *r = ring + (size_t)wp * NR * stride;
    int run[NR];
    Rv om[NR];
#pragma unroll
    for (int j = 0; j < NR; j++) {
        run[j] = st->rhs[j].running;
        om[j] = (Rv)st->rhs[j].omega;
    }
    // tiles of VEC_BLOCK sites walked by a persistent grid (persistent_grid), so the reduction's
    // per-block fence and ticket are paid once per block
    constexpr int P = BasePack<Rv, NR>::P;
    typedef PackIO<Rv, P> IO;
    typedef PackElem<Rv, P> PE;
    const int ntiles = (Vh + VEC_BLOCK - 1) / VEC_BLOCK;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int k = tile * VEC_BLOCK + threadIdx.x;
        double red[NR];
#pragma unroll
        for (int j = 0; j < NR; j++) red[j] = 0.0;
        if (k < Vh) {
#pragma unroll
            for (int q = 0; q < NR / P; q++) {
                int any = 0, all = 1;
#pragma unroll
                for (int i = 0; i < P; i++) {
                    any |= run[q * P + i];
                    all &= run[q * P + i];
                }
                if (!any) continue;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const size_t o = bidx<Rv, NR>(q * P, c, k, Vh) / P;  // pack element
                    cpx<Rv> rv[P], sv[P], keep[P];
                    IO::ld((const PE *)rprev + o, rv);
                    IO::ld((const PE *)s + o, sv);
                    if (!all) IO::ldc((const PE *)r + o, keep);  // a stopped RHS keeps its slot
#pragma unroll
                    for (int i = 0; i < P; i++) {
                        const int j = q * P + i;
                        if (run[j]) {
                            rv[i].re = rv[i].re + om[j] * sv[i].re;
                            rv[i].im = rv[i].im + om[j] * sv[i].im;
                            red[j] += dot2((double)rv[i].re, (double)rv[i].re, (double)rv[i].im, (double)rv[i].im);
                        } else {
                            rv[i] = keep[i];
                        }
                    }
                    IO::st((PE *)r + o, rv);
                }
            }
        }
        reduce_tile<NR>(red, partials, tile);
    }
    FinLambda<NR> fin{st};
    reduce_last<NR>(partials, ticket, ntiles * (VEC_BLOCK / RED_CHUNK), fin);
}

// p = r_m + gamma p (the base search direction; the shifted p_i and x_i are updated once per
// window by ms_flush_kernel)
template <typename Rv, int NR>
__global__ void __launch_bounds__(VEC_BLOCK) ms_update_kernel(int Vh, size_t stride, const typename MSVec<Rv>::E *__restrict__ ring,
                                                               typename MSVec<Rv>::E *p, MSState *st)
{
    typedef typename MSVec<Rv>::E E;
    constexpr int P = BasePack<Rv, NR>::P;
    typedef PackIO<Rv, P> IO;
    typedef PackElem<Rv, P> PE;
    if (*(volatile int *)&st->stop_k4) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Vh) return;
    const E *r = ring + (size_t)((*(volatile const int *)&st->wpos + MS_WIN - 1) % MS_WIN) * NR * stride;
#pragma unroll
    for (int q = 0; q < NR / P; q++) {
        int run[P], any = 0;
        Rv g[P];
#pragma unroll
        for (int i = 0; i < P; i++) {
            run[i] = st->rhs[q * P + i].running;
            g[i] = (Rv)st->rhs[q * P + i].gamma;
            any |= run[i];
        }
        if (!any) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const size_t o = bidx<Rv, NR>(q * P, c, k, Vh) / P;  // pack element
            cpx<Rv> rv[P], pv[P];
            IO::ld((const PE *)r + o, rv);
            IO::ldc((const PE *)p + o, pv);
#pragma unroll
            for (int i = 0; i < P; i++)
                if (run[i]) {  // a stopped RHS keeps its direction
                    pv[i].re = rv[i].re + g[i] * pv[i].re;
                    pv[i].im = rv[i].im + g[i] * pv[i].im;
                }
            IO::st((PE *)p + o, pv);
        }
    }
}

// End of a window of m = wpos iterations with residuals r_1..r_m (ring slots 0..m-1).  Over the
// window the per-iteration updates x_i -= om_k p_i, p_i = ze_k r_k + ga_k p_i compose to
//   x_i = X0_i - cx0 P0_i - sum_k cx_k r_k,   p_i = ca P0_i + sum_k cb_k r_k
// with P0_i, X0_i the stored vectors of the window start.  The first NR*nshift threads of every
// block derive (cx0, cx, ca, cb) of one (rhs, shift) from the recorded scalars into shared memory
// (skipping iterations where the shift was frozen), then every site applies them: each shifted
// vector is read and written once per window instead of once per iteration.
template <typename Rv, typename Rx, int NR>
__global__ void __launch_bounds__(VEC_BLOCK) ms_flush_kernel(int Vh, int nshift, size_t stride,
                                                              const typename MSVec<Rv>::E *__restrict__ ring,
                                                              typename MSVec<Rx>::E *ps, typename MSVec<Rx>::E *x,
                                                              double *partials, unsigned *ticket, MSState *st)
{
    typedef typename MSVec<Rx>::E E;
    __shared__ double s_cx0[NR * MS_MAX_SHIFT], s_ca[NR * MS_MAX_SHIFT];
    __shared__ double s_cx[NR * MS_MAX_SHIFT][MS_WIN], s_cb[NR * MS_MAX_SHIFT][MS_WIN];
    __shared__ int s_use[NR * MS_MAX_SHIFT];  // 0: nothing to do, 1: x only, 2: x and p
    const int wp = *(volatile const int *)&st->wpos;
    for (int t = threadIdx.x; t < NR * nshift; t += blockDim.x) {
        const int j = t / nshift, i = t % nshift;
        const MSRhs &q = st->rhs[j];
        double cx0 = 0.0, ca = 1.0, cx[MS_WIN], cb[MS_WIN];
        int any = 0;
        for (int m = 0; m < MS_WIN; m++) cx[m] = cb[m] = 0.0;
        for (int m = 0; m < wp; m++) {
            if (!q.h_act[i][m]) continue;
            any = 1;
            const double om = q.h_om[i][m], ga = q.h_ga[i][m];
            cx0 += om * ca;
            for (int l = 0; l < m; l++) cx[l] += om * cb[l];
            ca *= ga;
            for (int l = 0; l < m; l++) cb[l] *= ga;
            cb[m] = q.h_ze[i][m];
        }
        s_cx0[t] = cx0;
        s_ca[t] = ca;
        for (int m = 0; m < MS_WIN; m++) {
            s_cx[t][m] = cx[m];
            s_cb[t][m] = cb[m];
        }
        // p_i is written for every shift still active, also when the RHS stopped in this window:
        // a later phase may resume it from exactly this state
        s_use[t] = any ? (q.active_next[i] ? 2 : 1) : 0;
    }
    __syncthreads();
    constexpr int P = BasePack<Rv, NR>::P;
    typedef PackIO<Rv, P> IO;
    typedef PackElem<Rv, P> PE;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < Vh && wp > 0) {
        for (int q = 0; q < NR / P; q++) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                // the window's residuals of this site, read once (a pack of P right-hand sides per
                // load) and shared by every shift
                cpx<Rv> rp[MS_WIN][P];
#pragma unroll
                for (int m = 0; m < MS_WIN; m++)
                    if (m < wp) IO::ld((const PE *)(ring + (size_t)m * NR * stride) + bidx<Rv, NR>(q * P, c, k, Vh) / P, rp[m]);
#pragma unroll
                for (int l = 0; l < P; l++) {
                    const int j = q * P + l;
                    E rv[MS_WIN];
#pragma unroll
                    for (int m = 0; m < MS_WIN; m++)
                        if (m < wp) {
                            rv[m].x = (Rx)rp[m][l].re;
                            rv[m].y = (Rx)rp[m][l].im;
                        }
                    for (int i = 0; i < nshift; i++) {
                        const int t = j * nshift + i, use = s_use[t];
                        if (!use) continue;
                        const size_t o = (size_t)t * stride + (size_t)c * Vh + k;
                        const Rx x0 = (Rx)s_cx0[t], a0 = (Rx)s_ca[t];
                        const E p0 = ps[o];
                        E xv = x[o];
                        E pv;
                        xv.x = xv.x - x0 * p0.x;
                        xv.y = xv.y - x0 * p0.y;
                        pv.x = a0 * p0.x;
                        pv.y = a0 * p0.y;
#pragma unroll
                        for (int m = 0; m < MS_WIN; m++) {
                            if (m >= wp) break;
                            const Rx cx = (Rx)s_cx[t][m], cb = (Rx)s_cb[t][m];
                            xv.x = xv.x - cx * rv[m].x;
                            xv.y = xv.y - cx * rv[m].y;
                            pv.x = pv.x + cb * rv[m].x;
                            pv.y = pv.y + cb * rv[m].y;
                        }
                        x[o] = xv;
                        if (use == 2) ps[o] = pv;
                    }
                }
            }
        }
    }
    double none[1] = {0.0};
    FinWindow fin{st};
    reduce_finalize<1>(none, partials, ticket, fin);
}

// ------------------------------------------------------------------ precision-scheduled resumption
// The rounding error a sloppy iteration adds to the shifted systems is proportional to the
// residual at that iteration, and the shifted systems never see it corrected (only the base
// system is reliably updated).  So the mixed solver runs its first iterations in FP64, stops each
// right-hand side once |r| <= tau |b|, and resumes the same recurrences (same scalars, same
// shifted vectors) with FP32 base vectors and links: every later error is then tau times smaller.

// One thread: every RHS that has not reached the final target (and still has an active shift)
// runs again; the phase target becomes the final one and a new window starts.
static __global__ void ms_rearm_kernel(MSState *st)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int any = 0;
    for (int r = 0; r < st->nrhs; r++) {
        MSRhs &q = st->rhs[r];
        q.res = st->res;
        int nact = 0;
        for (int i = 0; i < st->nshift; i++) nact += q.active_next[i];
        const int go = st->status == 0 && isfinite(q.lambda) && q.b2 > 0.0 && sqrt(q.lambda) > st->res && nact > 0;
        q.running_next = go;
        q.ru_best = q.lambda;
        q.ru_stall = 0;
        any |= go;
    }
    st->tau = 0.0;
    st->stop = any ? 0 : 1;
    st->stop_k4 = 0;
    st->wpos = 0;
    st->ru_windows = 0;
    st->ru_now = 0;
}

// The current residual of every RHS (ring slot rslot of the previous phase) into the last slot of
// the new ring, and the base direction p, converted to the new phase's precision.
template <typename Rf, typename Rt, int NR>
__global__ void __launch_bounds__(VEC_BLOCK) ms_convert_kernel(int Vh, size_t stride, const typename MSVec<Rf>::E *__restrict__ ring_f,
                                                                const typename MSVec<Rf>::E *__restrict__ p_f,
                                                                typename MSVec<Rt>::E *ring_t, typename MSVec<Rt>::E *p_t,
                                                                const MSState *st)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Vh) return;
#pragma unroll
    for (int j = 0; j < NR; j++) {
        const int slot = st->rhs[j].rslot;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const size_t of = bidx<Rf, NR>(j, c, k, Vh), ot = bidx<Rt, NR>(j, c, k, Vh);
            const typename MSVec<Rf>::E rv = ring_f[(size_t)slot * NR * stride + of], pv = p_f[of];
            typename MSVec<Rt>::E a, b;
            a.x = (Rt)rv.x;
            a.y = (Rt)rv.y;
            b.x = (Rt)pv.x;
            b.y = (Rt)pv.y;
            ring_t[(size_t)(MS_WIN - 1) * NR * stride + ot] = a;
            p_t[ot] = b;
        }
    }
}

// One thread, after the window's flush: decides whether this window ends with a reliable update.
static __global__ void ms_ru_begin_kernel(MSState *st)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    st->ru_now = 0;
    if (st->stop) return;
    st->ru_windows++;
    int any = 0;
    for (int r = 0; r < st->nrhs; r++) any |= st->rhs[r].running_next;
    st->ru_now = any && (st->ru_windows % st->ru_every == 0);
}

// x0[j] = x_{j, i0(j)}: the FP64 base solution of every RHS, contiguous for the FP64 operator
template <int NR>
__global__ void __launch_bounds__(VEC_BLOCK) ms_gather_base_kernel(int Vh, int nshift, size_t stride, const double2 *__restrict__ x,
                                                                    double2 *x0, const MSState *st)
{
    if (!*(volatile const int *)&st->ru_now) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Vh) return;
#pragma unroll
    for (int j = 0; j < NR; j++) {
        const size_t src = (size_t)(j * nshift + st->rhs[j].i0) * stride;
#pragma unroll
        for (int c = 0; c < 3; c++) x0[j * stride + (size_t)c * Vh + k] = x[src + (size_t)c * Vh + k];
    }
}

// A right-hand side whose true base residual has not fallen by 4x (|r| by 2x) over
// MS_RU_STALL reliable updates, or has grown 4x above its best, has reached the rounding floor
// of the FP64 operator: past it the sloppy recurrence only follows rounding noise and diverges.
// It stops there (its solutions as they are) and is left to the refinement that follows.
constexpr int MS_RU_STALL = 16;

template <int NR>
struct FinMsRU {
    MSState *st;
    __device__ void operator()(const double *tot) const
    {
        if (threadIdx.x != 0) return;
        int any = 0;
        for (int r = 0; r < NR; r++) {
            MSRhs &q = st->rhs[r];
            if (!q.running_next) continue;
            if (!isfinite(tot[r])) {
                st->status = 2;
                q.running_next = 0;
                continue;
            }
            q.delta = tot[r];
            q.lambda = tot[r];
            if (tot[r] < 0.25 * q.ru_best) {
                q.ru_best = tot[r];
                q.ru_stall = 0;
            } else if (++q.ru_stall >= MS_RU_STALL || tot[r] > 4.0 * q.ru_best) {
                q.running_next = 0;
            }
            any |= q.running_next;
        }
        for (int r = NR; r < st->nrhs; r++) any |= st->rhs[r].running_next;
        if (!any) st->stop = 1;
        st->ru_count++;
    }
};

// Reliable update of every running RHS: r = b - t with t = (M^dag M + sigma_0) x0 computed in
// FP64 (the true residual of the base system) replaces the window's last residual, and the
// base direction is re-synchronised with the FP64 shifted direction of the base shift (both
// follow the same recurrence; the sloppy copy drifts by rounding).  |r|^2 becomes delta.
template <typename Rv, int NR>
__global__ void __launch_bounds__(VEC_BLOCK) ms_ru_resid_kernel(int Vh, int nshift, size_t stride, const double2 *__restrict__ b,
                                                                 const double2 *__restrict__ t, const double2 *__restrict__ ps,
                                                                 typename MSVec<Rv>::E *ring, typename MSVec<Rv>::E *p,
                                                                 double *partials, unsigned *ticket, MSState *st)
{
    typedef typename MSVec<Rv>::E E;
    if (!*(volatile const int *)&st->ru_now) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double red[NR];
#pragma unroll
    for (int j = 0; j < NR; j++) red[j] = 0.0;
    if (k < Vh) {
#pragma unroll
        for (int j = 0; j < NR; j++) {
            if (!st->rhs[j].running_next) continue;
            const size_t pbase = (size_t)(j * nshift + st->rhs[j].i0) * stride;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const size_t o = j * stride + (size_t)c * Vh + k, ob = bidx<Rv, NR>(j, c, k, Vh);
                const double2 bv = b[o], tv = t[o], pv = ps[pbase + (size_t)c * Vh + k];
                const double re = bv.x - tv.x, im = bv.y - tv.y;
                red[j] += dot2(re, re, im, im);
                E e, f;
                e.x = (Rv)re;
                e.y = (Rv)im;
                f.x = (Rv)pv.x;
                f.y = (Rv)pv.y;
                ring[(size_t)(MS_WIN - 1) * NR * stride + ob] = e;
                p[ob] = f;
            }
        }
    }
    FinMsRU<NR> fin{st};
    reduce_finalize<NR>(red, partials, ticket, fin);
}

}  // namespace rhmc
