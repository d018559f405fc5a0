// msolve_mixed.cu -- the mixed-precision batched multi-shift solver and the extern "C"
// multi-shift entry points.
//
// Mixed mode (no counterpart in the reference, which picks FP32 or FP64 per call by the
// requested residual, lib/Action/Inverter/cu_inverter.cc:45-60):
//   Phase A  multi-shift CG (msolve.cuh) with FP32 links/vectors, all right-hand sides
//            batched (every link load serves every RHS), base operator M^dag M + sigma_min,
//            until every shift reaches tol_A |b| (FP64 scalars and reductions).
//   Phase B  every (RHS, shift) system is refined by FP32 CG inside an FP64 defect correction:
//            once a system's FP32 residual has dropped by a factor delta since its last
//            update it waits; every n_ru iterations the waiting systems add their FP32
//            correction to the FP64 solution, recompute the residual b - (M^dag M + sigma) x
//            in FP64 with FP64 links and restart their FP32 CG from it (keeping the old search
//            direction across the update diverged for kappa ~ 1e5).  A system is finished only
//            when that FP64 true residual is <= the target.  Systems are sorted by shift and
//            refined in batches of up to 8 that share link loads.
// With fmt = RHMC_LINKS_F16_12 phase A runs on FP32 12-real links and phase B's sloppy CG keeps
// its links, residual, search direction and Dslash intermediates in half precision with a
// per-site scale (H16S; the correction accumulates in FP32), which halves its memory traffic.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "capi_util.h"
#include "context.h"
#include "kernels.h"
#include "msolve.cuh"
#include "solver.h"

namespace rhmc {

constexpr int RB_MAX = 8;
// windows (of MS_WIN iterations) between reliable updates of the FP32 multi-shift phase
constexpr int MX_RU_WINDOWS = 4;

struct ResidCoef {
    double coef[8];  // mass^2 + sigma of each batched system
};

struct RBState {
    int stop;         // every system converged (or failed)
    int status;       // 0 ok, 2 non-finite
    int nsys;
    int first;        // the next reliable update is the initial one (sets p = r)
    int ru_count;
    int iters;        // sloppy iterations performed
    int any_pending;  // some system waits for a reliable update
    int ru_max;       // force an update after this many sloppy iterations
    double delta2;    // update when |r_sloppy|^2 <= delta2 |r at last update|^2
    double tgt[RB_MAX];
    double rr[RB_MAX];     // |r_sloppy|^2
    double rr_ru[RB_MAX];  // |r|^2 at the last reliable update
    double alpha[RB_MAX], beta[RB_MAX];
    double r2true[RB_MAX];
    int conv[RB_MAX];
    int pending[RB_MAX];   // waiting for the next reliable update
    int hold[RB_MAX];      // skipped by the sloppy iteration
    int since[RB_MAX];     // sloppy iterations since the last update
};

// x += xs (FP64 += the sloppy accumulator X), xs = 0, for systems not yet converged
template <int NR, typename X>
__global__ void __launch_bounds__(VEC_BLOCK) rb_accum_kernel(int Vh, size_t stride, double2 *x, X *xs, const RBState *st)
{
    if (*(volatile const int *)&st->stop || !*(volatile const int *)&st->any_pending) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Vh) return;
#pragma unroll
    for (int j = 0; j < NR; j++) {
        if (st->conv[j] || !st->pending[j]) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const size_t o = j * stride + (size_t)c * Vh + k;
            double2 xv = x[o];
            X d = xs[o];
            xv.x += (double)d.x;
            xv.y += (double)d.y;
            x[o] = xv;
            d.x = 0;
            d.y = 0;
            xs[o] = d;
        }
    }
}

template <int NR>
struct FinRU {
    RBState *st;
    __device__ void operator()(const double *tot) const
    {
        if (threadIdx.x != 0) return;
        int all = 1;
        for (int j = 0; j < NR; j++) {
            if (st->conv[j]) continue;
            if (st->pending[j]) {
                const double r2 = tot[j];
                st->pending[j] = 0;
                st->since[j] = 0;
                if (!isfinite(r2)) {
                    st->status = 2;
                    st->conv[j] = 1;
                    continue;
                }
                st->r2true[j] = r2;
                st->rr[j] = r2;
                st->rr_ru[j] = r2;
                if (sqrt(r2) <= st->tgt[j]) st->conv[j] = 1;
            }
            all &= st->conv[j];
        }
        st->first = 0;
        st->ru_count++;
        st->any_pending = 0;
        if (all) st->stop = 1;
    }
};

// r = b - coef*x - t (FP64), rs = r in the sloppy storage S, |r|^2; the search direction is
// restarted from it (p = rs)
template <int NR, class S>
__global__ void __launch_bounds__(VEC_BLOCK) rb_resid_kernel(int Vh, size_t stride, size_t sstride, const double2 *__restrict__ b,
                                                              const double2 *__restrict__ x, const double2 *__restrict__ t,
                                                              typename S::elem *rs, typename S::elem *p, ResidCoef co,
                                                              double *partials, unsigned *ticket, RBState *st)
{
    if (*(volatile const int *)&st->stop || !*(volatile const int *)&st->any_pending) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double red[NR];
#pragma unroll
    for (int j = 0; j < NR; j++) red[j] = 0.0;
    if (k < Vh) {
#pragma unroll
        for (int j = 0; j < NR; j++) {
            if (st->conv[j] || !st->pending[j]) continue;
            vec3<double> r;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const size_t o = j * stride + (size_t)c * Vh + k;
                const double2 bv = b[o], xv = x[o], tv = t[o];
                const double re = bv.x - co.coef[j] * xv.x - tv.x, im = bv.y - co.coef[j] * xv.y - tv.y;
                red[j] += dot2(re, re, im, im);
                r.c[c] = mk<double>(re, im);
            }
            S::template store<double>(rs + j * sstride, Vh, k, r);
            S::template store<double>(p + j * sstride, Vh, k, r);
        }
    }
    FinRU<NR> fin{st};
    reduce_finalize<NR>(red, partials, ticket, fin);
}

template <int NR>
struct FinRBAlpha {
    RBState *st;
    __device__ void operator()(const double *tot) const
    {
        if (threadIdx.x != 0) return;
        for (int j = 0; j < NR; j++) {
            const double pap = tot[j];
            st->hold[j] = st->pending[j];
            const int skip = st->conv[j] || st->hold[j];
            st->alpha[j] = (skip || !(pap > 0.0)) ? 0.0 : st->rr[j] / pap;
            if (!skip && !isfinite(pap)) st->status = 2;
        }
        st->iters++;
    }
};

template <int NR>
struct FinRBBeta {
    RBState *st;
    __device__ void operator()(const double *tot) const
    {
        if (threadIdx.x != 0) return;
        for (int j = 0; j < NR; j++) {
            if (st->conv[j] || st->hold[j]) { st->beta[j] = 0.0; continue; }
            const double rn = tot[j];
            st->beta[j] = (st->rr[j] > 0.0) ? rn / st->rr[j] : 0.0;
            st->rr[j] = rn;
            st->since[j]++;
            // update after a drop by delta, after ru_max iterations, or when the FP32 iteration
            // stops making progress (its residual above 4x the last true one)
            if (rn <= st->delta2 * st->rr_ru[j] || st->since[j] >= st->ru_max || !isfinite(rn) || rn > 4.0 * st->rr_ru[j]) {
                st->pending[j] = 1;
                st->any_pending = 1;
            }
        }
    }
};

// xs += alpha p ; rs -= alpha Ap ; |rs|^2  (p, Ap, rs in the sloppy storage S; xs of type X)
template <int NR, class S, typename X>
__global__ void __launch_bounds__(VEC_BLOCK) rb_xr_kernel(int Vh, size_t stride, size_t sstride, X *xs, typename S::elem *rs,
                                                           const typename S::elem *__restrict__ p,
                                                           const typename S::elem *__restrict__ ap, double *partials,
                                                           unsigned *ticket, RBState *st)
{
    typedef typename S::real Rs;
    if (*(volatile const int *)&st->stop) return;
    // tiles of VEC_BLOCK sites walked by a persistent grid (persistent_grid)
    const int ntiles = (Vh + VEC_BLOCK - 1) / VEC_BLOCK;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int k = tile * VEC_BLOCK + threadIdx.x;
        double red[NR];
#pragma unroll
        for (int j = 0; j < NR; j++) red[j] = 0.0;
        if (k < Vh) {
#pragma unroll
            for (int j = 0; j < NR; j++) {
                if (st->conv[j] || st->hold[j]) continue;
                const Rs a = (Rs)st->alpha[j];
                const vec3<Rs> pv = S::template load<Rs>(p + j * sstride, Vh, k),
                               av = S::template load<Rs>(ap + j * sstride, Vh, k);
                vec3<Rs> rv = S::template load<Rs>(rs + j * sstride, Vh, k);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const size_t o = j * stride + (size_t)c * Vh + k;
                    X xv = xs[o];
                    xv.x += a * pv.c[c].re;
                    xv.y += a * pv.c[c].im;
                    xs[o] = xv;
                    rv.c[c].re -= a * av.c[c].re;
                    rv.c[c].im -= a * av.c[c].im;
                    red[j] += dot2((double)rv.c[c].re, (double)rv.c[c].re, (double)rv.c[c].im, (double)rv.c[c].im);
                }
                S::template store<Rs>(rs + j * sstride, Vh, k, rv);
            }
        }
        reduce_tile<NR>(red, partials, tile);
    }
    FinRBBeta<NR> fin{st};
    reduce_last<NR>(partials, ticket, ntiles * (VEC_BLOCK / RED_CHUNK), fin);
}

// p = rs + beta p
template <int NR, class S>
__global__ void __launch_bounds__(VEC_BLOCK) rb_p_kernel(int Vh, size_t sstride, const typename S::elem *__restrict__ rs,
                                                          typename S::elem *p, const RBState *st)
{
    typedef typename S::real Rs;
    if (*(volatile const int *)&st->stop) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Vh) return;
#pragma unroll
    for (int j = 0; j < NR; j++) {
        if (st->conv[j] || st->hold[j]) continue;
        const Rs be = (Rs)st->beta[j];
        const vec3<Rs> rv = S::template load<Rs>(rs + j * sstride, Vh, k);
        vec3<Rs> pv = S::template load<Rs>(p + j * sstride, Vh, k);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            pv.c[c].re = rv.c[c].re + be * pv.c[c].re;
            pv.c[c].im = rv.c[c].im + be * pv.c[c].im;
        }
        S::template store<Rs>(p + j * sstride, Vh, k, pv);
    }
}

// ------------------------------------------------------------------ Phase B driver
template <class LF, int NR>
static int rb_group(rhmc_ctx *c, const LF &lf, const double *coef, const double *tgt, double2 *xg, const double2 *bg,
                    int max_iter, int n_ru, long *iters_out, int *ru_out, double ru_delta)
{
    AuxScope aux_scope(c);
    cudaStream_t s_ = c->aux;
    const int Vh = (int)c->Vh;
    const size_t stride = 3 * (size_t)Vh;  // FP64 fields and the accumulator xs
    void *xs, *rs, *p, *ap, *h, *h64, *t64, *stv, *part, *tick;
    typedef typename LF::real Rs;
    typedef typename LF::store S;  // sloppy storage of rs, p, ap, h
    typedef typename S::elem E;
    typedef typename std::conditional<std::is_same<S, F64S>::value, double2, float2>::type X;
    const size_t sstride = (size_t)S::planes * Vh;
    const size_t vs = sstride * sizeof(E), vx = stride * sizeof(X), v64 = stride * sizeof(double2);
    CK(c->ws.get("rb_xs", NR * vx, &xs));
    CK(c->ws.get("rb_rs", NR * vs, &rs));
    CK(c->ws.get("rb_p", NR * vs, &p));
    CK(c->ws.get("rb_ap", NR * vs, &ap));
    CK(c->ws.get("rb_h", NR * vs, &h));
    CK(c->ws.get("rb_h64", NR * v64, &h64));
    CK(c->ws.get("rb_t64", NR * v64, &t64));
    CK(c->ws.get("rb_state", sizeof(RBState), &stv));
    const int gv = grid_for(Vh, VEC_BLOCK);
    CK(c->ws.get("rb_partials", (size_t)red_chunks(Vh) * 2 * NR * sizeof(double), &part));
    CK(c->ws.get("rb_tickets", 4 * sizeof(unsigned), &tick));
    L64_18 l64;
    links_f64_18(c, &l64);
    RBState *st = (RBState *)stv;
    unsigned *tk = (unsigned *)tick;
    double *pt = (double *)part;

    RBState h0;
    memset(&h0, 0, sizeof(h0));
    h0.nsys = NR;
    h0.first = 1;
    h0.any_pending = 1;
    h0.delta2 = ru_delta * ru_delta;
    h0.ru_max = 2000;
    for (int j = 0; j < NR; j++) {
        h0.tgt[j] = tgt[j];
        h0.pending[j] = 1;
    }
    CK(cudaMemcpyAsync(st, &h0, sizeof(h0), cudaMemcpyHostToDevice, s_));
    CK(cudaMemsetAsync(tk, 0, 4 * sizeof(unsigned), s_));
    CK(cudaMemsetAsync(xs, 0, NR * vx, s_));

    ResidCoef co;
    for (int j = 0; j < 8; j++) co.coef[j] = coef[j < NR ? j : 0];

    // FP64 M^dag M pieces of the reliable update
    DslashArgs<L64_18, NR, NoFin> d1;
    memset(&d1, 0, sizeof(d1));
    d1.g = c->g; d1.p_out = 1; d1.links = l64; d1.in = xg; d1.out = (double2 *)h64; d1.stride = stride; d1.beta = 0.5;
    d1.stop = &st->stop;
    d1.run_if = &st->any_pending;
    DslashArgs<L64_18, NR, NoFin> d2 = d1;
    d2.p_out = 0; d2.in = (const double2 *)h64; d2.out = (double2 *)t64; d2.beta = -0.5;
    // sloppy operator
    DslashArgs<LF, NR, NoFin> s1;
    memset(&s1, 0, sizeof(s1));
    s1.g = c->g; s1.p_out = 1; s1.links = lf; s1.in = (const E *)p; s1.out = (E *)h; s1.stride = sstride;
    s1.beta = (Rs)0.5; s1.stop = &st->stop;
    DslashArgs<LF, NR, FinRBAlpha<NR>> s2;
    memset(&s2, 0, sizeof(s2));
    s2.g = c->g; s2.p_out = 0; s2.links = lf; s2.in = (const E *)h; s2.out = (E *)ap; s2.y = (const E *)p;
    s2.stride = sstride; s2.beta = (Rs)-0.5; s2.use_alphas = 1;
    for (int j = 0; j < NR; j++) s2.alphas[j] = (Rs)coef[j];
    s2.partials = pt; s2.ticket = tk + 1; s2.fin.st = st; s2.stop = &st->stop;

    struct Key {
        int kind, link_reals, link_bytes, nr, n_ru, vh;
        const void *links, *links64, *xs, *rs, *p, *ap, *h, *h64, *t64, *st, *pt, *tk, *xg, *bg;
        double coef[RB_MAX];
        cudaStream_t stream;
        int cand[3];  // launch shapes of the captured Dslash instantiations
    } key;
    memset(&key, 0, sizeof(key));
    // launch shapes (tuned now, outside the capture, when unknown)
    key.cand[0] = dslash_candidate<L64_18, NR, false, false>(c->g, l64, s_);
    key.cand[1] = dslash_candidate<LF, NR, false, false>(c->g, lf, s_);
    key.cand[2] = dslash_candidate<LF, NR, true, true>(c->g, lf, s_);
    key.kind = 2; key.link_reals = LF::reals; key.link_bytes = (int)sizeof(typename LF::real); key.nr = NR;
    key.n_ru = n_ru; key.vh = Vh; key.links = lf.p; key.links64 = l64.p; key.xs = xs; key.rs = rs; key.p = p;
    key.ap = ap; key.h = h; key.h64 = h64; key.t64 = t64; key.st = st; key.pt = pt; key.tk = tk; key.xg = xg;
    key.bg = bg; key.stream = s_;
    for (int j = 0; j < NR; j++) key.coef[j] = coef[j];
    const std::string kb = key_bytes(key);
    cudaGraphExec_t exec = c->graphs.find(kb);
    cudaError_t ce = cudaSuccess;
    if (!exec) {
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        rb_accum_kernel<NR, X><<<gv, VEC_BLOCK, 0, s_>>>(Vh, stride, xg, (X *)xs, st);
        dslash_launch_cand<L64_18, NR, false, false, NoFin>(key.cand[0], d1, Vh, s_);
        dslash_launch_cand<L64_18, NR, false, false, NoFin>(key.cand[0], d2, Vh, s_);
        rb_resid_kernel<NR, S><<<gv, VEC_BLOCK, 0, s_>>>(Vh, stride, sstride, bg, xg, (const double2 *)t64, (E *)rs, (E *)p,
                                                             co, pt, tk, st);
        for (int it = 0; it < n_ru; it++) {
            dslash_launch_cand<LF, NR, false, false, NoFin>(key.cand[1], s1, Vh, s_);
            dslash_launch_cand<LF, NR, true, true, FinRBAlpha<NR>>(key.cand[2], s2, Vh, s_);
            rb_xr_kernel<NR, S, X><<<persistent_grid((const void *)rb_xr_kernel<NR, S, X>, VEC_BLOCK, gv), VEC_BLOCK, 0,
                                     s_>>>(Vh, stride, sstride, (X *)xs, (E *)rs, (const E *)p, (const E *)ap, pt, tk + 2, st);
            rb_p_kernel<NR, S><<<gv, VEC_BLOCK, 0, s_>>>(Vh, sstride, (const E *)rs, (E *)p, st);
        }
        ce = cudaStreamEndCapture(s_, &graph);
        if (ce != cudaSuccess) return cuda_fail(ce, "refine capture");
        ce = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return cuda_fail(ce, "refine instantiate");
        c->graphs.put(kb, exec);
    }

    const long max_rep = max_iter / n_ru + 2;
    long rep = 0;
    int seen = 0;
    const int prc = replay_until_stop(c, exec, s_, &st->stop, max_rep, &rep, &seen, "refine loop");
    c->launches += rep * (4 + 4 * (long)n_ru);
    if (prc) return prc;
    RBState hs;
    CK(cudaMemcpy(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost));
    *iters_out += hs.iters;
    *ru_out += hs.ru_count;
    if (hs.status == 2) return fail(RHMC_ERR_NONFINITE, "refinement: non-finite reduction");
    if (!hs.stop) return fail(RHMC_ERR_MAXITER, "refinement: iteration cap %d reached", max_iter);
    return RHMC_OK;
}

template <class LF>
static int rb_group_n(rhmc_ctx *c, const LF &lf, int n, const double *coef, const double *tgt, double2 *xg, const double2 *bg,
                      int max_iter, int n_ru, long *iters, int *ru, double ru_delta)
{
    switch (n) {
    case 1: return rb_group<LF, 1>(c, lf, coef, tgt, xg, bg, max_iter, n_ru, iters, ru, ru_delta);
    case 2: return rb_group<LF, 2>(c, lf, coef, tgt, xg, bg, max_iter, n_ru, iters, ru, ru_delta);
    case 3: return rb_group<LF, 3>(c, lf, coef, tgt, xg, bg, max_iter, n_ru, iters, ru, ru_delta);
    case 4: return rb_group<LF, 4>(c, lf, coef, tgt, xg, bg, max_iter, n_ru, iters, ru, ru_delta);
    case 8: return rb_group<LF, 8>(c, lf, coef, tgt, xg, bg, max_iter, n_ru, iters, ru, ru_delta);
    default: return fail(RHMC_ERR_ARG, "bad refinement batch %d", n);
    }
}

// Refine all (rhs, shift) systems of x (FP64 internal [nrhs][nshift]) to |b - A_sigma x| <= res.
template <class LF>
static int refine_all(rhmc_ctx *c, const LF &lf, int nshift, const double *shifts, int nrhs, double res, int max_iter,
                      double2 *x, const double2 *b, long *iters, int *ru, double ru_delta, int max_batch = RB_MAX,
                      const double *skip_below = nullptr, int *nsys = nullptr)
{
    const size_t stride = 3 * (size_t)c->Vh;
    const size_t v64 = stride * sizeof(double2);
    void *xg, *bg;
    CK(c->ws.get("rb_xg", RB_MAX * v64, &xg));
    CK(c->ws.get("rb_bg", RB_MAX * v64, &bg));
    std::vector<int> order;
    for (int q = 0; q < nshift * nrhs; q++)
        if (!skip_below || skip_below[q] > res) order.push_back(q);
    std::stable_sort(order.begin(), order.end(), [&](int a, int bq) { return shifts[a] < shifts[bq]; });
    if (nsys) *nsys = (int)order.size();
    const double m2 = c->mass * c->mass;
    size_t g0 = 0;
    while (g0 < order.size()) {
        const size_t left = order.size() - g0;
        int n = left >= 8 ? 8 : (left >= 4 ? 4 : (int)left);  // instantiated batch widths
        if (n > max_batch) n = max_batch;
        double coef[RB_MAX], tgt[RB_MAX];
        for (int j = 0; j < n; j++) {
            const int q = order[g0 + j];
            coef[j] = m2 + shifts[q];  // shifts [nrhs][nshift], q = r * nshift + i
            tgt[j] = res;
            CK(cudaMemcpyAsync((double2 *)xg + j * stride, x + (size_t)q * stride, v64, cudaMemcpyDeviceToDevice, c->stream));
            CK(cudaMemcpyAsync((double2 *)bg + j * stride, b + (size_t)(q / nshift) * stride, v64, cudaMemcpyDeviceToDevice,
                               c->stream));
        }
        // iterations between reliable-update stages (systems that need none skip the stage)
        const double kappa = (16.0 + coef[0]) / coef[0];
        const int n_ru = kappa > 1e3 ? 16 : 8;
        int rc = rb_group_n(c, lf, n, coef, tgt, (double2 *)xg, (const double2 *)bg, max_iter, n_ru, iters, ru, ru_delta);
        if (rc) return rc;
        for (int j = 0; j < n; j++) {
            const int q = order[g0 + j];
            CK(cudaMemcpyAsync(x + (size_t)q * stride, (double2 *)xg + j * stride, v64, cudaMemcpyDeviceToDevice, c->stream));
        }
        g0 += n;
    }
    return RHMC_OK;
}

int msolve_mixed(rhmc_ctx *c, int fmt, int nshift, const double *shifts, int nrhs, double res, int max_iter, double tolA,
                 double ru_delta, double2 *x, const double2 *b, rhmc_msolve_info *info)
{
    auto t0 = std::chrono::steady_clock::now();
    std::vector<double> base(nrhs);  // each RHS iterates on its smallest pole
    for (int r = 0; r < nrhs; r++) {
        base[r] = shifts[(size_t)r * nshift];
        for (int i = 1; i < nshift; i++) base[r] = std::min(base[r], shifts[(size_t)r * nshift + i]);
    }
    MSolveArgs A;
    A.nshift = nshift;
    A.nrhs = nrhs;
    A.shift = shifts;
    A.base = base.data();
    A.max_iter = max_iter;
    A.stop_on_frozen = 1;
    A.chunk = 8;
    A.b = b;
    MSolveInfo mi;
    memset(&mi, 0, sizeof(mi));
    std::vector<double> tgt(nshift);
    std::vector<double> tr;  // FP64 true residuals after the multi-shift phase
    int it_hi[8] = {0};      // iterations of each RHS in the FP64 part of the precision schedule
    int rc;
    const bool f64a = fmt_is_f64(fmt);
    if (f64a) {
        // Phase A in FP64 (compressed links when fmt is 12-real), straight into x
        for (double &t : tgt) t = res;
        A.tgt = tgt.data();
        A.res_base = res;
        A.x = x;
        rc = msolve_shifted(c, fmt, A, &mi);
        if (rc && rc != RHMC_ERR_MAXITER) return rc;
        tr.resize((size_t)nshift * nrhs);
        rc = true_residuals(c, nshift, shifts, nrhs, x, b, tr.data());
        if (rc) return rc;
        for (double &v : tr) v = std::sqrt(v);
    } else {
        // Precision schedule: FP64 (12-real links) until |r| <= tol_A |b| for every RHS, then the
        // same recurrences resumed with FP32 links and base vectors, FP64 shifted vectors and a
        // reliable update of the base system every MX_RU_WINDOWS windows, to the final target.
        for (double &t : tgt) t = res;
        A.tgt = tgt.data();
        A.res_base = res;
        A.x = x;
        A.tau = tolA;
        rc = msolve_shifted(c, RHMC_LINKS_F64_12, A, &mi);
        if (rc && rc != RHMC_ERR_MAXITER) return rc;
        for (int r = 0; r < nrhs && r < 8; r++) it_hi[r] = mi.iters[r];
        if (rc == RHMC_OK) {
            A.fresh = 0;
            A.tau = 0.0;
            A.ru_every = MX_RU_WINDOWS;
            // half refinement follows an FP32 multi-shift on 12-real links
            rc = msolve_shifted(c, fmt == RHMC_LINKS_F16_12 ? RHMC_LINKS_F32_12 : fmt, A, &mi);
            if (rc && rc != RHMC_ERR_MAXITER) return rc;
        }
        tr.resize((size_t)nshift * nrhs);
        rc = true_residuals(c, nshift, shifts, nrhs, x, b, tr.data());
        if (rc) return rc;
        for (double &v : tr) v = std::sqrt(v);
    }
    const double t_a = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    long it_b = 0;
    int ru = 0, nsys = 0;
    // refinement: half links and spinors for F16_12, else FP32 sloppy links of the matching width
    if (fmt == RHMC_LINKS_F16_12) {
        L16_12 lf;
        links_f16_12(c, &lf);
        rc = refine_all(c, lf, nshift, shifts, nrhs, res, max_iter, x, b, &it_b, &ru, ru_delta, RB_MAX,
                        tr.empty() ? nullptr : tr.data(), &nsys);
    } else if (fmt == RHMC_LINKS_F32_18 || fmt == RHMC_LINKS_F64_18) {
        L32_18 lf;
        links_f32_18(c, &lf);
        rc = refine_all(c, lf, nshift, shifts, nrhs, res, max_iter, x, b, &it_b, &ru, ru_delta, RB_MAX,
                        tr.empty() ? nullptr : tr.data(), &nsys);
    } else {
        L32_12 lf;
        links_f32_12(c, &lf);
        rc = refine_all(c, lf, nshift, shifts, nrhs, res, max_iter, x, b, &it_b, &ru, ru_delta, RB_MAX,
                        tr.empty() ? nullptr : tr.data(), &nsys);
    }
    CK(cudaStreamSynchronize(c->stream));
    if (info) {
        info->status = rc;
        for (int r = 0; r < nrhs && r < 8; r++) info->iters[r] = mi.iters[r];
        info->refine_iters = it_b;
        info->reliable_updates = ru;
        info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        info->seconds_phase_a = t_a;
        info->systems_refined = nsys;
        for (int r = 0; r < nrhs && r < 8; r++) info->iters_fp64 += f64a ? mi.iters[r] : it_hi[r];
        info->ms_reliable_updates = f64a ? 0 : mi.ru_count;
    }
    return rc;
}

}  // namespace rhmc

using namespace rhmc;

// multi-shift iteration counts of right-hand sides first..first+n-1 into info (the per-RHS
// array holds the first 8; the total and the maximum cover all of them)
static void add_iters(rhmc_msolve_info *info, int first, const int *it, int n)
{
    if (!info) return;
    for (int j = 0; j < n; j++) {
        if (first + j < 8) info->iters[first + j] = it[j];
        info->iters_total += it[j];
        if (it[j] > info->iters_max) info->iters_max = it[j];
    }
}

// sh: the pole sets [nrhs][nshift]
static int msolve_fp64(rhmc_ctx *c, const rhmc_msolve_params *P, const double *sh, double2 *x, const double2 *b,
                       rhmc_msolve_info *info)
{
    const size_t stride = 3 * (size_t)c->Vh;
    std::vector<double> tgt(P->nshift, P->residual), zero(MS_MAX_RHS, 0.0);
    int done = 0, rc = RHMC_OK;
    auto t0 = std::chrono::steady_clock::now();
    while (done < P->nrhs) {
        const int left = P->nrhs - done;
        const int n = left >= 8 ? 8 : (left >= 4 ? 4 : left);
        MSolveArgs A;
        A.nshift = P->nshift;
        A.nrhs = n;
        A.shift = sh + (size_t)done * P->nshift;
        A.base = zero.data();  // the reference iterates on M^dag M itself
        A.tgt = tgt.data();
        A.res_base = P->residual;
        A.max_iter = P->max_iter;
        A.stop_on_frozen = 1;
        A.chunk = 8;
        A.b = b + (size_t)done * stride;
        A.x = x + (size_t)done * P->nshift * stride;
        MSolveInfo mi;
        memset(&mi, 0, sizeof(mi));
        rc = msolve_shifted(c, P->fmt, A, &mi);
        add_iters(info, done, mi.iters, n);
        if (rc) break;
        done += n;
    }
    long it_b = 0;
    int ru = 0, nsys = 0;
    cudaStreamSynchronize(c->stream);
    const double t_a = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc == RHMC_OK && P->certify) {
        // FP64 defect correction of every system whose FP64 true residual is above target
        std::vector<double> tr((size_t)P->nshift * P->nrhs);
        rc = true_residuals(c, P->nshift, sh, P->nrhs, x, b, tr.data());
        for (double &v : tr) v = std::sqrt(v);
        if (rc == RHMC_OK) {
            L64_18 lf;
            links_f64_18(c, &lf);
            rc = refine_all(c, lf, P->nshift, sh, P->nrhs, P->residual, P->max_iter, x, b, &it_b, &ru, 0.05, 1, tr.data(), &nsys);
        }
        cudaStreamSynchronize(c->stream);
    }
    if (info) {
        info->status = rc;
        info->refine_iters = it_b;
        info->reliable_updates = ru;
        info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        info->seconds_phase_a = t_a;
        info->systems_refined = nsys;
    }
    return rc;
}

// The reference's single-precision path (cuda_shifted_inverter, lib/Cuda/cuda_inverter.cu:647-857):
// the same recurrences with FP32 links and base vectors and FP64 scalars.  The shifted solutions
// and directions are accumulated in FP64 (the reference keeps them in FP32), which removes their
// storage rounding from the true residual; they are written straight into x.
static int msolve_fp32(rhmc_ctx *c, const rhmc_msolve_params *P, const double *sh, double2 *x, const double2 *b,
                       rhmc_msolve_info *info)
{
    const size_t stride = 3 * (size_t)c->Vh;
    std::vector<double> tgt(P->nshift, P->residual), zero(MS_MAX_RHS, 0.0);
    auto t0 = std::chrono::steady_clock::now();
    int done = 0, rc = RHMC_OK;
    while (done < P->nrhs) {
        const int left = P->nrhs - done;
        const int n = left >= 8 ? 8 : (left >= 4 ? 4 : left);
        MSolveArgs A;
        A.nshift = P->nshift;
        A.nrhs = n;
        A.shift = sh + (size_t)done * P->nshift;
        A.base = zero.data();
        A.tgt = tgt.data();
        A.res_base = P->residual;
        A.max_iter = P->max_iter;
        A.stop_on_frozen = 1;
        A.chunk = 8;
        A.b = b + (size_t)done * stride;
        A.x = x + (size_t)done * P->nshift * stride;
        MSolveInfo mi;
        memset(&mi, 0, sizeof(mi));
        rc = msolve_shifted(c, P->fmt, A, &mi);
        add_iters(info, done, mi.iters, n);
        if (rc) break;
        done += n;
    }
    CK(cudaStreamSynchronize(c->stream));
    if (info) {
        info->status = rc;
        info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return rc;
}

extern "C" {

int rhmc_msolve(rhmc_ctx *c, const rhmc_msolve_params *P, double *x, const double *b, rhmc_msolve_info *info)
{
    if (!c || !P || !x || !b || (!P->shifts && !P->rhs_shifts)) return fail(RHMC_ERR_ARG, "null argument");
    if (P->nshift < 1 || P->nshift > MS_MAX_SHIFT) return fail(RHMC_ERR_ARG, "nshift must be in [1, %d]", MS_MAX_SHIFT);
    if (P->nrhs < 1) return fail(RHMC_ERR_ARG, "nrhs must be >= 1");
    if (P->max_iter < 1) return fail(RHMC_ERR_ARG, "max_iter must be >= 1");
    // the pole set of every RHS: rhs_shifts [nrhs][nshift], or shifts for all of them
    std::vector<double> sh((size_t)P->nrhs * P->nshift);
    for (int r = 0; r < P->nrhs; r++)
        for (int i = 0; i < P->nshift; i++)
            sh[(size_t)r * P->nshift + i] = P->rhs_shifts ? P->rhs_shifts[(size_t)r * P->nshift + i] : P->shifts[i];
    for (double v : sh)
        if (!(v >= 0.0)) return fail(RHMC_ERR_ARG, "shifts must be >= 0");
    if (info) memset(info, 0, sizeof(*info));
    if (P->mode == RHMC_MSOLVE_FP64) {
        if (P->fmt != RHMC_LINKS_F64_18 && P->fmt != RHMC_LINKS_F64_12) return fail(RHMC_ERR_ARG, "FP64 mode needs FP64 links");
        return msolve_fp64(c, P, sh.data(), (double2 *)x, (const double2 *)b, info);
    }
    if (P->mode == RHMC_MSOLVE_FP32) {
        if (P->fmt != RHMC_LINKS_F32_18 && P->fmt != RHMC_LINKS_F32_12) return fail(RHMC_ERR_ARG, "FP32 mode needs FP32 links");
        return msolve_fp32(c, P, sh.data(), (double2 *)x, (const double2 *)b, info);
    }
    if (P->mode == RHMC_MSOLVE_MIXED) {
        if (P->fmt < 0 || P->fmt > RHMC_LINKS_F16_12) return fail(RHMC_ERR_ARG, "bad link format %d", P->fmt);
        // the hand-over of the precision schedule: the caller's, or 1e-3 |b| but at most
        // MS_TAU_REACH above the target (negative: automatic)
        const double tolA = P->tol_phase_a > 0 ? P->tol_phase_a : -1e-3;
        const double rud = (P->ru_delta > 0 && P->ru_delta < 1) ? P->ru_delta : 0.05;
        // batches of 8, 4, 3, 2 or 1 right-hand sides (the widths the kernels are built for)
        const size_t stride = 3 * (size_t)c->Vh;
        int done = 0, rc = RHMC_OK;
        rhmc_msolve_info agg, part;
        memset(&agg, 0, sizeof(agg));
        while (done < P->nrhs && rc == RHMC_OK) {
            const int left = P->nrhs - done;
            const int n = left >= 8 ? 8 : (left >= 4 ? 4 : left);
            memset(&part, 0, sizeof(part));
            rc = msolve_mixed(c, P->fmt, P->nshift, sh.data() + (size_t)done * P->nshift, n, P->residual, P->max_iter, tolA, rud,
                              (double2 *)x + (size_t)done * P->nshift * stride, (const double2 *)b + (size_t)done * stride, &part);
            add_iters(&agg, done, part.iters, n);
            agg.refine_iters += part.refine_iters;
            agg.reliable_updates += part.reliable_updates;
            agg.seconds += part.seconds;
            agg.seconds_phase_a += part.seconds_phase_a;
            agg.systems_refined += part.systems_refined;
            agg.iters_fp64 += part.iters_fp64;
            agg.ms_reliable_updates += part.ms_reliable_updates;
            done += n;
        }
        agg.status = rc;
        if (info) *info = agg;
        return rc;
    }
    return fail(RHMC_ERR_ARG, "bad solver mode %d", P->mode);
}

int rhmc_msolve_host(rhmc_ctx *c, const rhmc_msolve_params *P, double *x, const double *b, rhmc_msolve_info *info)
{
    if (!c || !P || !x || !b) return fail(RHMC_ERR_ARG, "null argument");
    const size_t stride = 3 * (size_t)c->Vh;
    const size_t nb = (size_t)P->nrhs, nx = (size_t)P->nrhs * P->nshift;
    void *bi, *xi, *tmp;
    CK(c->ws.get("mh_b", nb * stride * sizeof(double2), &bi));
    CK(c->ws.get("mh_x", nx * stride * sizeof(double2), &xi));
    CK(c->ws.get("mh_tmp", (nx > nb ? nx : nb) * stride * sizeof(double2), &tmp));
    CK(cudaMemcpyAsync(tmp, b, nb * stride * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    launch_spinor_to_internal(c, RHMC_LINKS_F64_18, bi, (const double *)tmp, (int)nb);
    int rc = rhmc_msolve(c, P, (double *)xi, (const double *)bi, info);
    if (rc) return rc;
    launch_spinor_from_internal(c, RHMC_LINKS_F64_18, (double *)tmp, xi, (int)nx);
    CK(cudaMemcpyAsync(x, tmp, nx * stride * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return RHMC_OK;
}

int rhmc_true_residuals(rhmc_ctx *c, int nshift, const double *shifts, int nrhs, const double *x, const double *b, double *out)
{
    if (!c || !shifts || !x || !b || !out || nshift < 1 || nrhs < 1) return fail(RHMC_ERR_ARG, "bad argument");
    std::vector<double> sh((size_t)nrhs * nshift);
    for (int r = 0; r < nrhs; r++)
        for (int i = 0; i < nshift; i++) sh[(size_t)r * nshift + i] = shifts[i];
    int rc = true_residuals(c, nshift, sh.data(), nrhs, (const double2 *)x, (const double2 *)b, out);
    if (rc) return rc;
    for (int i = 0; i < nshift * nrhs; i++) out[i] = std::sqrt(out[i]);
    return RHMC_OK;
}

}  // extern "C"
