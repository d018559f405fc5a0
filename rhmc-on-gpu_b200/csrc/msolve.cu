// msolve.cu -- host orchestration of the multi-shift CG (msolve.cuh): workspace, CUDA-graph
// capture of one delayed-update window of iterations, device-flag polling, and the extern "C" entry points.
#include <cmath>
#include <cstring>
#include <vector>

#include "capi_util.h"
#include "context.h"
#include "kernels.h"
#include "msolve.cuh"
#include "solver.h"

namespace rhmc {

static int vec_grid(rhmc_ctx *c) { return grid_for(c->Vh, VEC_BLOCK); }

template <class LF, int NR>
static int ms_run_nr(rhmc_ctx *c, const LF &lf, const MSolveArgs &A, MSolveInfo *info)
{
    AuxScope aux_scope(c);
    cudaStream_t s_ = c->aux;
    typedef typename LF::real Rv;
    typedef typename SpinorT<Rv>::elem E;
    const int Vh = (int)c->Vh;
    const size_t stride = 3 * (size_t)Vh;
    const size_t vbytes = stride * sizeof(E);
    const int S = A.nshift;
    void *r, *p, *h, *s, *ps, *stv, *part, *tick;
    CK(c->ws.get("ms_r", (size_t)MS_WIN * NR * vbytes, &r));  // ring of the window's residuals [slot][rhs]
    CK(c->ws.get("ms_p", NR * vbytes, &p));
    CK(c->ws.get("ms_h", NR * vbytes, &h));
    CK(c->ws.get("ms_s", NR * vbytes, &s));
    CK(c->ws.get("ms_ps", (size_t)NR * S * vbytes, &ps));
    CK(c->ws.get("ms_state", sizeof(MSState), &stv));
    const int gv = vec_grid(c);
    // the grids of this configuration's two Dslash launches
    const int gd1 = grid_for(Vh, DslashCfg<LF, NR, false>::block), gd2 = grid_for(Vh, DslashCfg<LF, NR, true>::block);
    CK(c->ws.get("ms_partials", (size_t)red_chunks(Vh) * 2 * NR * sizeof(double), &part));
    CK(c->ws.get("ms_tickets", 4 * sizeof(unsigned), &tick));
    int *hflag = c->hflags;
    MSState *st = (MSState *)stv;
    unsigned *tk = (unsigned *)tick;
    double *pt = (double *)part;
    E *xs = (E *)A.x;

    // host-side constants of the state
    MSState h0;
    memset(&h0, 0, sizeof(h0));
    h0.nshift = S;
    h0.nrhs = NR;
    h0.max_iter = A.max_iter;
    h0.stop_on_frozen = A.stop_on_frozen;
    h0.res = A.res_base;
    for (int i = 0; i < S; i++) h0.tgt[i] = A.tgt[i];
    for (int r = 0; r < NR; r++)
        for (int i = 0; i < S; i++) h0.rhs[r].shift[i] = A.shift[(size_t)r * S + i] - A.base[r];
    h0.wpos = 0;
    CK(cudaMemcpyAsync(st, &h0, sizeof(MSState), cudaMemcpyHostToDevice, s_));
    CK(cudaMemsetAsync(tk, 0, 4 * sizeof(unsigned), s_));

    ms_init_kernel<Rv, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, S, stride, (const double2 *)A.b, (E *)r, (E *)p, (E *)ps, xs,
                                                            pt, tk, st);
    c->launches++;
    CK(cudaGetLastError());

    // D_oe and D_eo launch arguments
    DslashArgs<LF, NR, NoFin> a1;
    memset(&a1, 0, sizeof(a1));
    a1.g = c->g;
    a1.p_out = 1;
    a1.links = lf;
    a1.in = (const E *)p;
    a1.out = (E *)h;
    a1.stride = stride;
    a1.beta = (Rv)0.5;
    a1.stop = &st->stop;
    a1.stop_set = &st->stop_k4;
    DslashArgs<LF, NR, FinAlpha<NR>> a2;
    memset(&a2, 0, sizeof(a2));
    a2.g = c->g;
    a2.p_out = 0;
    a2.links = lf;
    a2.in = (const E *)h;
    a2.out = (E *)s;
    a2.y = (const E *)p;
    a2.stride = stride;
    a2.alpha = (Rv)(c->mass * c->mass + A.base[0]);
    a2.use_alphas = 1;  // every RHS iterates its own base operator M^dag M + base[r]
    for (int r = 0; r < NR; r++) a2.alphas[r] = (Rv)(c->mass * c->mass + A.base[r]);
    a2.beta = (Rv)-0.5;
    a2.partials = pt;
    a2.ticket = tk + 1;
    a2.fin.st = st;
    a2.stop = &st->stop;

    const int chunk = MS_WIN;  // one graph replay = one delayed-update window
    struct Key {
        int kind, link_reals, link_bytes, nr, chunk, nshift, vh;
        const void *links, *r, *p, *h, *s, *ps, *xs, *pt, *tk, *st;
        double alpha[MS_MAX_RHS];
        cudaStream_t stream;
    } key;
    memset(&key, 0, sizeof(key));
    key.kind = 4; key.link_reals = LF::reals; key.link_bytes = (int)sizeof(typename LF::real); key.nr = NR;
    key.chunk = chunk; key.nshift = S; key.vh = Vh; key.links = lf.p; key.r = r; key.p = p; key.h = h; key.s = s;
    key.ps = ps; key.xs = xs; key.pt = pt; key.tk = tk; key.st = st; key.stream = s_;
    for (int r = 0; r < NR; r++) key.alpha[r] = (double)a2.alphas[r];
    const std::string kb = key_bytes(key);
    cudaError_t ce = cudaSuccess;
    cudaGraphExec_t exec = c->graphs.find(kb);
    if (!exec) {
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        for (int it = 0; it < chunk; it++) {
            dslash_kernel<LF, NR, false, false, NoFin><<<gd1, DslashCfg<LF, NR, false>::block, 0, s_>>>(a1);
            dslash_kernel<LF, NR, true, true, FinAlpha<NR>><<<gd2, DslashCfg<LF, NR, true>::block, 0, s_>>>(a2);
            ms_resid_kernel<Rv, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, stride, (E *)r, (const E *)s, pt, tk + 2, st);
            ms_update_kernel<Rv, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, stride, (const E *)r, (E *)p, st);
        }
        ms_flush_kernel<Rv, NR><<<gv, VEC_BLOCK, 0, s_>>>(Vh, S, stride, (const E *)r, (E *)ps, xs, pt, tk + 3, st);
        ce = cudaStreamEndCapture(s_, &graph);
        if (ce != cudaSuccess) return cuda_fail(ce, "msolve capture");
        ce = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return cuda_fail(ce, "msolve instantiate");
        c->graphs.put(kb, exec);
    }

    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    const long max_chunks = (A.max_iter + chunk - 1) / chunk + 2;
    long launched = 0;
    bool done = false;
    hflag[0] = hflag[1] = 0;
    for (long ch = 0; ch < max_chunks && !done; ch++) {
        ce = cudaGraphLaunch(exec, s_);
        if (ce != cudaSuccess) break;
        launched++;
        cudaMemcpyAsync(&hflag[ch & 1], &st->stop, sizeof(int), cudaMemcpyDeviceToHost, s_);
        cudaEventRecord(ev[ch & 1], s_);
        if (ch >= 1) {
            cudaEventSynchronize(ev[(ch - 1) & 1]);
            if (hflag[(ch - 1) & 1]) done = true;
        }
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s_);
    c->launches += launched * (chunk * 4 + 1);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (ce != cudaSuccess) return cuda_fail(ce, "msolve loop");

    MSState hs;
    CK(cudaMemcpy(&hs, st, sizeof(MSState), cudaMemcpyDeviceToHost));
    if (info) {
        info->status = hs.status;
        info->graph_replays = launched;
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
    case 1: return ms_run_nr<LF, 1>(c, lf, A, info);
    case 2: return ms_run_nr<LF, 2>(c, lf, A, info);
    case 3: return ms_run_nr<LF, 3>(c, lf, A, info);
    case 4: return ms_run_nr<LF, 4>(c, lf, A, info);
    case 8: return ms_run_nr<LF, 8>(c, lf, A, info);
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
