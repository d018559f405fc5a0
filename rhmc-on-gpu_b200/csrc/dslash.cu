// dslash.cu -- instantiation and dispatch of the Dslash kernels (dslash.cuh).
#include "context.h"
#include "dslash.cuh"
#include "kernels.h"

namespace rhmc {

bool fmt_is_f64(int fmt) { return fmt == RHMC_LINKS_F64_18 || fmt == RHMC_LINKS_F64_12; }

// the largest Dslash grid of any configuration (sizes the per-block reduction partials)
int dslash_grid(rhmc_ctx *c) { return grid_for(c->Vh, DSLASH_MIN_BLOCK); }

template <class LF, int NR>
static cudaError_t run(rhmc_ctx *c, const LF &lf, int p_out, void *out, const void *in, size_t stride, const void *y,
                       double alpha, double beta)
{
    typedef typename LF::real R;
    typedef typename LF::store::elem E;
    DslashArgs<LF, NR> a;
    memset(&a, 0, sizeof(a));
    a.g = c->g;
    a.p_out = p_out;
    a.links = lf;
    a.in = (const E *)in;
    a.out = (E *)out;
    a.y = (const E *)y;
    a.stride = stride;
    a.alpha = (R)alpha;
    a.beta = (R)beta;
    for (int r = 0; r < NR; r++) a.alphas[r] = (R)alpha;
    c->launches++;
    if (y) return dslash_launch<LF, NR, true, false, NoFin>(a, (int)c->Vh, c->stream);
    return dslash_launch<LF, NR, false, false, NoFin>(a, (int)c->Vh, c->stream);
}

// one launch of m in {1, 2, 3, 4, 8} right-hand sides
template <class LF>
static cudaError_t run_width(rhmc_ctx *c, const LF &lf, int p_out, void *out, const void *in, size_t stride, int m,
                             const void *y, double alpha, double beta)
{
    switch (m) {
    case 1: return run<LF, 1>(c, lf, p_out, out, in, stride, y, alpha, beta);
    case 2: return run<LF, 2>(c, lf, p_out, out, in, stride, y, alpha, beta);
    case 3: return run<LF, 3>(c, lf, p_out, out, in, stride, y, alpha, beta);
    case 4: return run<LF, 4>(c, lf, p_out, out, in, stride, y, alpha, beta);
    case 8: return run<LF, 8>(c, lf, p_out, out, in, stride, y, alpha, beta);
    default: return cudaErrorInvalidValue;
    }
}

// RHS packing w: launches of the widest built width <= w (8, 4, 3, 2, 1) until all n are done
template <class LF>
static cudaError_t run_packed(rhmc_ctx *c, const LF &lf, int p_out, void *out, const void *in, size_t stride, int n,
                              const void *y, double alpha, double beta, int w)
{
    typedef typename LF::store::elem E;
    int done = 0;
    while (done < n) {
        const int left = n - done < w ? n - done : w;
        const int m = left >= 8 ? 8 : (left >= 4 ? 4 : left);
        const cudaError_t e = run_width<LF>(c, lf, p_out, (E *)out + done * stride, (const E *)in + done * stride, stride, m,
                                            y ? (const E *)y + done * stride : nullptr, alpha, beta);
        if (e != cudaSuccess) return e;
        done += m;
    }
    return cudaSuccess;
}

// The RHS packings a call with n >= 5 right-hand sides can use (at most 8, 4 or 3 per launch); the
// tuned one is found by timing each on the call's own buffers (outputs are rewritten by the final
// launch, inputs only read), once per device, volume, link format, n and epilogue.
constexpr int DS_PACK[3] = {8, 4, 3};

template <class LF>
static cudaError_t run_n(rhmc_ctx *c, const LF &lf, int p_out, void *out, const void *in, size_t stride, int n, const void *y,
                         double alpha, double beta)
{
    if (n == 1 || n == 2 || n == 3 || n == 4) return run_width<LF>(c, lf, p_out, out, in, stride, n, y, alpha, beta);
    int pick = 0;
    if (autotune_override() >= 0) {
        pick = autotune_override();
    } else if (autotune_enabled()) {
        const std::string key = tune_key(c->Vh, std::string("pack ") + LF::name + " n=" + std::to_string(n) +
                                                    " y=" + std::to_string(y ? 1 : 0));
        pick = tune_get(key);
        if (pick < 0) {
            pick = 0;
            if (y != out && !stream_capturing(c->stream)) {
                cudaEvent_t e0 = nullptr, e1 = nullptr;
                float us[3] = {0, 0, 0};
                cudaError_t e = cudaEventCreate(&e0);
                if (e == cudaSuccess) e = cudaEventCreate(&e1);
                for (int w = 0; w < 3 && e == cudaSuccess; w++) {
                    e = run_packed<LF>(c, lf, p_out, out, in, stride, n, y, alpha, beta, DS_PACK[w]);  // warm-up
                    cudaEventRecord(e0, c->stream);
                    for (int r = 0; r < 3 && e == cudaSuccess; r++)
                        e = run_packed<LF>(c, lf, p_out, out, in, stride, n, y, alpha, beta, DS_PACK[w]);
                    cudaEventRecord(e1, c->stream);
                    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                    float ms = 0.f;
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                    us[w] = ms * 1e3f / 3.f;
                }
                if (e0) cudaEventDestroy(e0);
                if (e1) cudaEventDestroy(e1);
                if (e != cudaSuccess) return e;
                for (int w = 1; w < 3; w++)
                    if (us[w] < us[pick]) pick = w;
                const DsShape packs[3] = {{DS_PACK[0], 0}, {DS_PACK[1], 0}, {DS_PACK[2], 0}};
                tune_put(key, pick, us, packs, 3);
            }
        }
    }
    return run_packed<LF>(c, lf, p_out, out, in, stride, n, y, alpha, beta, DS_PACK[pick < 0 || pick > 2 ? 0 : pick]);
}

// FP64 18-real half-Dslash of one spinor in the reference's site-major layout (A64S) onto the
// output sites [k_lo, k_lo + k_count) only, on stream s (the host-buffer entry point pipelines
// its copies against these slabs)
cudaError_t launch_dslash_f64_range(rhmc_ctx *c, cudaStream_t s, int p_out, void *out, const void *in, int k_lo, int k_count)
{
    L64_18 l18;
    cudaError_t e = links_f64_18(c, &l18);
    if (e != cudaSuccess) return e;
    L64_18A lf;
    lf.p = l18.p;
    lf.Vh = l18.Vh;
    DslashArgs<L64_18A, 1> a;
    memset(&a, 0, sizeof(a));
    a.g = c->g;
    a.p_out = p_out;
    a.links = lf;
    a.in = (const double2 *)in;
    a.out = (double2 *)out;
    a.stride = 3 * (size_t)c->Vh;
    a.beta = 0.5;
    a.k_lo = k_lo;
    a.k_count = k_count;
    c->launches++;
    return dslash_launch<L64_18A, 1, false, false, NoFin>(a, k_count, s);
}

cudaError_t launch_dslash(rhmc_ctx *c, int fmt, int p_out, void *out, const void *in, size_t stride, int n,
                          const void *y, double alpha, double beta, double *partials, int *nblocks)
{
    if (partials) return cudaErrorInvalidValue;  // reductions go through the solver's own launches
    if (nblocks) *nblocks = dslash_grid(c);
    cudaError_t e = cudaSuccess;
    switch (fmt) {
    case RHMC_LINKS_F64_18: { L64_18 lf; e = links_f64_18(c, &lf); if (!e) e = run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta); break; }
    case RHMC_LINKS_F64_12: { L64_12 lf; e = links_f64_12(c, &lf); if (!e) e = run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta); break; }
    case RHMC_LINKS_F32_18: { L32_18 lf; e = links_f32_18(c, &lf); if (!e) e = run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta); break; }
    case RHMC_LINKS_F32_12: { L32_12 lf; e = links_f32_12(c, &lf); if (!e) e = run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta); break; }
    case RHMC_LINKS_F16_12: { L16_12 lf; e = links_f16_12(c, &lf); if (!e) e = run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta); break; }
    default: return cudaErrorInvalidValue;
    }
    return e;
}

}  // namespace rhmc
