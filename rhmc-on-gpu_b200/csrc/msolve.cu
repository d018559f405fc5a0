// msolve.cu -- host orchestration of the multi-shift CG (msolve.cuh): workspace, CUDA-graph
// capture of one delayed-update window of iterations, device-flag polling, the FP64-to-FP32
// precision schedule with reliable updates, and the FP64 true residuals.
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

static int vec_grid(rhmc_ctx *c) { return grid_for(c->Vh, VEC_BLOCK); }

int replay_until_stop(rhmc_ctx *c, cudaGraphExec_t exec, cudaStream_t s, const int *stop, long max_rep, long *replays,
                      int *stop_seen, const char *what)
{
    int *hflag = c->hflags;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaError_t ce = cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    long rep = 0;
    bool done = false;
    hflag[0] = hflag[1] = 0;
    for (; ce == cudaSuccess && rep < max_rep && !done; rep++) {
        ce = cudaGraphLaunch(exec, s);
        if (ce != cudaSuccess) break;
        ce = cudaMemcpyAsync(&hflag[rep & 1], stop, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaEventRecord(ev[rep & 1], s);
        if (ce == cudaSuccess && rep >= 1) {
            ce = cudaEventSynchronize(ev[(rep - 1) & 1]);
            if (ce == cudaSuccess && hflag[(rep - 1) & 1]) done = true;
        }
    }
    *replays = rep;
    const cudaError_t cs = cudaStreamSynchronize(s);
    if (ce == cudaSuccess) ce = cs;
    if (ce == cudaSuccess && !done && rep > 0) done = hflag[(rep - 1) & 1] != 0;
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    *stop_seen = done ? 1 : 0;
    if (ce != cudaSuccess) return cuda_fail(ce, what);
    return RHMC_OK;
}

// workspace slot name of a base vector set in elements of `bytes` bytes
static std::string vname(const char *base, size_t bytes) { return std::string(base) + std::to_string(bytes); }

// One phase of the multi-shift CG with links LF: base vectors (residual ring, p, h, s) in the
// links' precision, shifted solutions and directions always FP64.  A fresh phase starts from
// x_i = 0; a resumed phase continues the state a previous FP64 phase left (scalars, shifted
// vectors, and its base vectors converted to this precision), optionally with reliable updates.
template <class LF, int NR>
static int ms_phase(rhmc_ctx *c, const LF &lf, const MSolveArgs &A, MSolveInfo *info)
{
    AuxScope aux_scope(c);
    cudaStream_t s_ = c->aux;
    typedef typename LF::real Rv;
    typedef typename SpinorT<Rv>::elem E;
    const int Vh = (int)c->Vh;
    const size_t stride = 3 * (size_t)Vh;
    const size_t vbytes = stride * sizeof(E), v64 = stride * sizeof(double2);
    const int S = A.nshift;
    const bool ru = A.ru_every > 0;
    if (!A.fresh && sizeof(E) == sizeof(double2)) return fail(RHMC_ERR_ARG, "multi-shift: an FP64 phase cannot resume an FP64 phase");
    void *r, *p, *h, *s, *ps, *stv, *part, *tick;
    CK(c->ws.get(vname("ms_r", sizeof(E)), (size_t)MS_WIN * NR * vbytes, &r));  // ring of the window's residuals [slot][rhs]
    CK(c->ws.get(vname("ms_p", sizeof(E)), NR * vbytes, &p));
    CK(c->ws.get(vname("ms_h", sizeof(E)), NR * vbytes, &h));
    CK(c->ws.get(vname("ms_s", sizeof(E)), NR * vbytes, &s));
    CK(c->ws.get("ms_ps", (size_t)NR * S * v64, &ps));
    CK(c->ws.get("ms_state", sizeof(MSState), &stv));
    const int gv = vec_grid(c);
    CK(c->ws.get("ms_partials", (size_t)red_chunks(Vh) * 2 * NR * sizeof(double), &part));
    CK(c->ws.get("ms_tickets", 8 * sizeof(unsigned), &tick));
    MSState *st = (MSState *)stv;
    unsigned *tk = (unsigned *)tick;
    double *pt = (double *)part;
    double2 *xs = (double2 *)A.x;

    if (A.fresh) {
        MSState h0;
        memset(&h0, 0, sizeof(h0));
        h0.nshift = S;
        h0.nrhs = NR;
        h0.max_iter = A.max_iter;
        h0.stop_on_frozen = A.stop_on_frozen;
        h0.res = A.res_base;
        h0.tau = A.tau;
        h0.ru_every = A.ru_every;
        for (int i = 0; i < S; i++) h0.tgt[i] = A.tgt[i];
        for (int rr = 0; rr < NR; rr++) {
            int i0 = -1;  // the pole the RHS iterates on (reliable updates need it among the poles)
            for (int i = 0; i < S; i++) {
                h0.rhs[rr].shift[i] = A.shift[(size_t)rr * S + i] - A.base[rr];
                if (i0 < 0 && A.shift[(size_t)rr * S + i] == A.base[rr]) i0 = i;
            }
            if (ru && i0 < 0) return fail(RHMC_ERR_ARG, "multi-shift: reliable updates need the base shift among the poles");
            h0.rhs[rr].i0 = i0 < 0 ? 0 : i0;
        }
        h0.wpos = 0;
        CK(cudaMemcpyAsync(st, &h0, sizeof(MSState), cudaMemcpyHostToDevice, s_));
        CK(cudaMemsetAsync(tk, 0, 8 * sizeof(unsigned), s_));
        ms_init_kernel<Rv, double, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, S, stride, (const double2 *)A.b, (E *)r, (E *)p,
                                                                 (double2 *)ps, xs, pt, tk, st);
        c->launches++;
        CK(cudaGetLastError());
    } else {
        // resume the FP64 phase's state in this phase's precision
        void *r64, *p64;
        CK(c->ws.get(vname("ms_r", sizeof(double2)), (size_t)MS_WIN * NR * v64, &r64));
        CK(c->ws.get(vname("ms_p", sizeof(double2)), NR * v64, &p64));
        CK(cudaMemcpyAsync(&st->res, &A.res_base, sizeof(double), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(&st->ru_every, &A.ru_every, sizeof(int), cudaMemcpyHostToDevice, s_));
        ms_rearm_kernel<<<1, 32, 0, s_>>>(st);
        ms_convert_kernel<double, Rv, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, stride, (const double2 *)r64, (const double2 *)p64,
                                                                     (E *)r, (E *)p, st);
        c->launches += 2;
        CK(cudaGetLastError());
    }

    // D_oe and D_eo launch arguments, on the base vectors' packed layout (BasePack)
    typedef typename std::conditional<BasePack<Rv, NR>::P == 1, LF, LPack<LF, BasePack<Rv, NR>::P>>::type LFB;
    typedef typename LFB::store::elem EB;
    LFB lfb;
    static_cast<LF &>(lfb) = lf;
    DslashArgs<LFB, NR, NoFin> a1;
    memset(&a1, 0, sizeof(a1));
    a1.g = c->g;
    a1.p_out = 1;
    a1.links = lfb;
    a1.in = (const EB *)p;
    a1.out = (EB *)h;
    a1.stride = stride;
    a1.beta = (Rv)0.5;
    a1.stop = &st->stop;
    a1.stop_set = &st->stop_k4;
    DslashArgs<LFB, NR, FinAlpha<NR>> a2;
    memset(&a2, 0, sizeof(a2));
    a2.g = c->g;
    a2.p_out = 0;
    a2.links = lfb;
    a2.in = (const EB *)h;
    a2.out = (EB *)s;
    a2.y = (const EB *)p;
    a2.stride = stride;
    a2.alpha = (Rv)(c->mass * c->mass + A.base[0]);
    a2.use_alphas = 1;  // every RHS iterates its own base operator M^dag M + base[r]
    for (int rr = 0; rr < NR; rr++) a2.alphas[rr] = (Rv)(c->mass * c->mass + A.base[rr]);
    a2.beta = (Rv)-0.5;
    a2.partials = pt;
    a2.ticket = tk + 1;
    a2.fin.st = st;
    a2.stop = &st->stop;

    // reliable update: t = (M^dag M + base) x0 with FP64 12-real links, x0 the FP64 base solutions
    L64_12 l64;
    void *x0 = nullptr, *h64 = nullptr, *t64 = nullptr;
    DslashArgs<L64_12, NR, NoFin> u1, u2;
    memset(&u1, 0, sizeof(u1));
    memset(&u2, 0, sizeof(u2));
    if (ru) {
        cudaError_t e = links_f64_12(c, &l64);
        if (e != cudaSuccess) return cuda_fail(e, "links");
        // the FP64 phase's base vectors are free once resumed: they hold x0, D_oe x0 and t
        CK(c->ws.get(vname("ms_p", sizeof(double2)), NR * v64, &x0));
        CK(c->ws.get(vname("ms_h", sizeof(double2)), NR * v64, &h64));
        CK(c->ws.get(vname("ms_s", sizeof(double2)), NR * v64, &t64));
        u1.g = c->g; u1.p_out = 1; u1.links = l64; u1.in = (const double2 *)x0; u1.out = (double2 *)h64; u1.stride = stride;
        u1.beta = 0.5; u1.run_if = &st->ru_now;
        u2 = u1;
        u2.p_out = 0; u2.in = (const double2 *)h64; u2.out = (double2 *)t64; u2.y = (const double2 *)x0; u2.beta = -0.5;
        u2.use_alphas = 1;
        for (int rr = 0; rr < NR; rr++) u2.alphas[rr] = c->mass * c->mass + A.base[rr];
    }

    const int chunk = MS_WIN;  // one graph replay = one delayed-update window
    struct Key {
        int kind, link_reals, link_bytes, nr, chunk, nshift, vh, ru_every;
        const void *links, *links64, *r, *p, *h, *s, *ps, *xs, *pt, *tk, *st, *x0, *h64, *t64, *b;
        double alpha[MS_MAX_RHS];
        cudaStream_t stream;
        int cand[4];  // launch shapes of the captured Dslash instantiations
    } key;
    memset(&key, 0, sizeof(key));
    // launch shapes (tuned now, outside the capture, when unknown)
    key.cand[0] = dslash_candidate<LFB, NR, false, false>(c->g, lfb, s_);
    key.cand[1] = dslash_candidate<LFB, NR, true, true>(c->g, lfb, s_);
    if (ru) {
        key.cand[2] = dslash_candidate<L64_12, NR, false, false>(c->g, l64, s_);
        key.cand[3] = dslash_candidate<L64_12, NR, true, false>(c->g, l64, s_);
    }
    key.kind = 4; key.link_reals = LF::reals; key.link_bytes = (int)sizeof(typename LF::real); key.nr = NR;
    key.chunk = chunk; key.nshift = S; key.vh = Vh; key.ru_every = A.ru_every; key.links = lf.p; key.r = r; key.p = p;
    key.h = h; key.s = s; key.ps = ps; key.xs = xs; key.pt = pt; key.tk = tk; key.st = st; key.stream = s_;
    if (ru) {
        key.links64 = l64.p; key.x0 = x0; key.h64 = h64; key.t64 = t64; key.b = A.b;
    }
    for (int rr = 0; rr < NR; rr++) key.alpha[rr] = (double)a2.alphas[rr];
    const std::string kb = key_bytes(key);
    cudaError_t ce = cudaSuccess;
    cudaGraphExec_t exec = c->graphs.find(kb);
    if (!exec) {
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        for (int it = 0; it < chunk; it++) {
            dslash_launch_cand<LFB, NR, false, false, NoFin>(key.cand[0], a1, Vh, s_);
            dslash_launch_cand<LFB, NR, true, true, FinAlpha<NR>>(key.cand[1], a2, Vh, s_);
            ms_resid_kernel<Rv, NR><<<persistent_grid((const void *)ms_resid_kernel<Rv, NR>, VEC_BLOCK, gv), VEC_BLOCK, 0,
                                      s_>>>(Vh, stride, (E *)r, (const E *)s, pt, tk + 2, st);
            ms_update_kernel<Rv, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, stride, (const E *)r, (E *)p, st);
        }
        ms_flush_kernel<Rv, double, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, S, stride, (const E *)r, (double2 *)ps, xs, pt, tk + 3, st);
        if (ru) {
            ms_ru_begin_kernel<<<1, 32, 0, s_>>>(st);
            ms_gather_base_kernel<NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, S, stride, xs, (double2 *)x0, st);
            dslash_launch_cand<L64_12, NR, false, false, NoFin>(key.cand[2], u1, Vh, s_);
            dslash_launch_cand<L64_12, NR, true, false, NoFin>(key.cand[3], u2, Vh, s_);
            ms_ru_resid_kernel<Rv, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, S, stride, (const double2 *)A.b, (const double2 *)t64,
                                                                  (const double2 *)ps, (E *)r, (E *)p, pt, tk + 4, st);
        }
        ce = cudaStreamEndCapture(s_, &graph);
        if (ce != cudaSuccess) return cuda_fail(ce, "msolve capture");
        ce = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return cuda_fail(ce, "msolve instantiate");
        c->graphs.put(kb, exec);
    }

    const long max_chunks = (A.max_iter + chunk - 1) / chunk + 2;
    long launched = 0;
    int seen = 0;
    const int prc = replay_until_stop(c, exec, s_, &st->stop, max_chunks, &launched, &seen, "msolve loop");
    c->launches += launched * (chunk * 4 + 1 + (ru ? 5 : 0));
    if (prc) return prc;

    MSState hs;
    CK(cudaMemcpy(&hs, st, sizeof(MSState), cudaMemcpyDeviceToHost));
    if (info) {
        info->status = hs.status;
        info->graph_replays += launched;
        info->ru_count = hs.ru_count;
        for (int j = 0; j < NR; j++) {
            info->iters[j] = hs.rhs[j].iter;
            info->lambda[j] = hs.rhs[j].lambda;
            info->b2[j] = hs.rhs[j].b2;
        }
    }
    if (hs.status == 2) return fail(RHMC_ERR_NONFINITE, "multi-shift CG: non-finite reduction");
    if (hs.status == 1) return fail(RHMC_ERR_MAXITER, "multi-shift CG: iteration cap %d reached", A.max_iter);
    return RHMC_OK;
}

template <class LF>
static int ms_run(rhmc_ctx *c, const LF &lf, const MSolveArgs &A, MSolveInfo *info)
{
    switch (A.nrhs) {
    case 1: return ms_phase<LF, 1>(c, lf, A, info);
    case 2: return ms_phase<LF, 2>(c, lf, A, info);
    case 3: return ms_phase<LF, 3>(c, lf, A, info);
    case 4: return ms_phase<LF, 4>(c, lf, A, info);
    case 8: return ms_phase<LF, 8>(c, lf, A, info);
    default: return fail(RHMC_ERR_ARG, "nrhs must be 1, 2, 3, 4 or 8 (got %d)", A.nrhs);
    }
}

int msolve_shifted(rhmc_ctx *c, int fmt, const MSolveArgs &A, MSolveInfo *info)
{
    if (A.nshift < 1 || A.nshift > MS_MAX_SHIFT) return fail(RHMC_ERR_ARG, "nshift must be in [1, %d]", MS_MAX_SHIFT);
    if (A.nrhs < 1 || A.nrhs > MS_MAX_RHS) return fail(RHMC_ERR_ARG, "nrhs must be in [1, %d]", MS_MAX_RHS);
    cudaError_t e;
    switch (fmt) {
    case RHMC_LINKS_F64_18: { L64_18 lf; e = links_f64_18(c, &lf); if (e) return cuda_fail(e, "links"); return ms_run(c, lf, A, info); }
    case RHMC_LINKS_F64_12: { L64_12 lf; e = links_f64_12(c, &lf); if (e) return cuda_fail(e, "links"); return ms_run(c, lf, A, info); }
    case RHMC_LINKS_F32_18: { L32_18 lf; e = links_f32_18(c, &lf); if (e) return cuda_fail(e, "links"); return ms_run(c, lf, A, info); }
    case RHMC_LINKS_F32_12: { L32_12 lf; e = links_f32_12(c, &lf); if (e) return cuda_fail(e, "links"); return ms_run(c, lf, A, info); }
    default: return fail(RHMC_ERR_ARG, "bad link format %d", fmt);
    }
}

// ------------------------------------------------------------------ true residuals (FP64)
struct ResidSys {
    int rhs[8];
    double coef[8];
};

// partial |b_rhs(j) - coef_j x_j - t_j|^2, j < J, with t_j = -Deo Doe x_j
__global__ void __launch_bounds__(VEC_BLOCK) resid_norm_kernel(int Vh, size_t stride, int J, ResidSys sys,
                                                                const double2 *__restrict__ b, const double2 *__restrict__ x,
                                                                const double2 *__restrict__ t, double *partials)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double red[8];
#pragma unroll
    for (int j = 0; j < 8; j++) red[j] = 0.0;
    if (k < Vh) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (j >= J) break;
            for (int c = 0; c < 3; c++) {
                const size_t o = (size_t)c * Vh + k;
                const double2 bv = b[sys.rhs[j] * stride + o], xv = x[j * stride + o], tv = t[j * stride + o];
                const double re = bv.x - sys.coef[j] * xv.x - tv.x, im = bv.y - sys.coef[j] * xv.y - tv.y;
                red[j] += re * re + im * im;
            }
        }
    }
    __shared__ double smem[8 * 32];
    block_sum<8>(red, smem);
    if (threadIdx.x == 0)
        for (int j = 0; j < J; j++) partials[(size_t)blockIdx.x * 8 + j] = red[j];
}

int true_residuals(rhmc_ctx *c, int nshift, const double *shifts, int nrhs, const double2 *x, const double2 *b, double *out)
{
    const int Vh = (int)c->Vh;
    const size_t stride = 3 * (size_t)Vh;
    void *h, *t, *part;
    CK(c->ws.get("tr_h", 8 * stride * sizeof(double2), &h));
    CK(c->ws.get("tr_t", 8 * stride * sizeof(double2), &t));
    const int gv = vec_grid(c);
    CK(c->ws.get("tr_part", (size_t)gv * 8 * sizeof(double), &part));
    std::vector<double> hp((size_t)gv * 8);
    const int total = nrhs * nshift;
    for (int j0 = 0; j0 < total; j0 += 8) {
        const int J = total - j0 < 8 ? total - j0 : 8;
        ResidSys sys;
        for (int j = 0; j < 8; j++) {
            const int q = j0 + (j < J ? j : 0);
            sys.rhs[j] = q / nshift;
            sys.coef[j] = c->mass * c->mass + shifts[q];  // [nrhs][nshift], q = r * nshift + i
        }
        const double2 *xj = x + (size_t)j0 * stride;
        cudaError_t e = launch_dslash(c, RHMC_LINKS_F64_18, 1, h, xj, stride, J, nullptr, 0.0, 0.5, nullptr, nullptr);
        if (e == cudaSuccess) e = launch_dslash(c, RHMC_LINKS_F64_18, 0, t, h, stride, J, nullptr, 0.0, -0.5, nullptr, nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "true_residuals");
        resid_norm_kernel<<<gv, VEC_BLOCK, 0, c->stream>>>(Vh, stride, J, sys, b, xj, (const double2 *)t, (double *)part);
        c->launches++;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hp.data(), part, (size_t)gv * 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int j = 0; j < J; j++) {
            double s = 0.0;
            for (int g = 0; g < gv; g++) s += hp[(size_t)g * 8 + j];
            out[j0 + j] = s;
        }
    }
    return RHMC_OK;
}

}  // namespace rhmc
