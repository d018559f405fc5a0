// dslash.cu -- instantiation and dispatch of the Dslash kernels (dslash.cuh).
#include "context.h"
#include "dslash.cuh"
#include "kernels.h"

namespace rhmc {

bool fmt_is_f64(int fmt) { return fmt == RHMC_LINKS_F64_18 || fmt == RHMC_LINKS_F64_12; }

// the largest Dslash grid of any configuration (sizes the per-block reduction partials)
int dslash_grid(rhmc_ctx *c) { return grid_for(c->Vh, DSLASH_MIN_BLOCK); }

template <class LF, int NR>
static void run(rhmc_ctx *c, const LF &lf, int p_out, void *out, const void *in, size_t stride, const void *y,
                double alpha, double beta, double *partials)
{
    typedef typename LF::real R;
    typedef typename LF::store::elem E;
    DslashArgs<LF, NR> a;
    a.g = c->g;
    a.p_out = p_out;
    a.links = lf;
    a.in = (const E *)in;
    a.out = (E *)out;
    a.y = (const E *)y;
    a.stride = stride;
    a.alpha = (R)alpha;
    a.beta = (R)beta;
    a.use_alphas = 0;
    for (int r = 0; r < NR; r++) a.alphas[r] = (R)alpha;
    a.partials = partials;
    a.ticket = nullptr;
    a.stop = nullptr;
    a.stop_set = nullptr;
    a.run_if = nullptr;
    constexpr int B = DslashCfg<LF, NR, false>::block;
    const int grid = grid_for(c->Vh, B);
    if (y) dslash_kernel<LF, NR, true, false, NoFin><<<grid, B, 0, c->stream>>>(a);
    else dslash_kernel<LF, NR, false, false, NoFin><<<grid, B, 0, c->stream>>>(a);
    c->launches++;
}

template <class LF>
static void run_n(rhmc_ctx *c, const LF &lf, int p_out, void *out, const void *in, size_t stride, int n, const void *y,
                  double alpha, double beta, double *partials)
{
    switch (n) {
    case 1: run<LF, 1>(c, lf, p_out, out, in, stride, y, alpha, beta, partials); break;
    case 2: run<LF, 2>(c, lf, p_out, out, in, stride, y, alpha, beta, partials); break;
    case 3: run<LF, 3>(c, lf, p_out, out, in, stride, y, alpha, beta, partials); break;
    case 4: run<LF, 4>(c, lf, p_out, out, in, stride, y, alpha, beta, partials); break;
    case 8: run<LF, 8>(c, lf, p_out, out, in, stride, y, alpha, beta, partials); break;
    default: {
        // split into supported widths
        typedef typename LF::store::elem E;
        int done = 0;
        while (done < n) {
            int m = n - done >= 8 ? 8 : (n - done >= 4 ? 4 : n - done);
            run_n<LF>(c, lf, p_out, (E *)out + done * stride, (const E *)in + done * stride, stride, m,
                      y ? (const E *)y + done * stride : nullptr, alpha, beta, nullptr);
            done += m;
        }
    }
    }
}

cudaError_t launch_dslash(rhmc_ctx *c, int fmt, int p_out, void *out, const void *in, size_t stride, int n,
                          const void *y, double alpha, double beta, double *partials, int *nblocks)
{
    if (partials) return cudaErrorInvalidValue;  // reductions go through the solver's own launches
    if (nblocks) *nblocks = dslash_grid(c);
    cudaError_t e = cudaSuccess;
    switch (fmt) {
    case RHMC_LINKS_F64_18: { L64_18 lf; e = links_f64_18(c, &lf); if (!e) run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta, partials); break; }
    case RHMC_LINKS_F64_12: { L64_12 lf; e = links_f64_12(c, &lf); if (!e) run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta, partials); break; }
    case RHMC_LINKS_F32_18: { L32_18 lf; e = links_f32_18(c, &lf); if (!e) run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta, partials); break; }
    case RHMC_LINKS_F32_12: { L32_12 lf; e = links_f32_12(c, &lf); if (!e) run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta, partials); break; }
    case RHMC_LINKS_F16_12: { L16_12 lf; e = links_f16_12(c, &lf); if (!e) run_n(c, lf, p_out, out, in, stride, n, y, alpha, beta, partials); break; }
    default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace rhmc
