// dslash.cuh -- the even/odd staggered hopping term on sm_100a.
//
// Half-Dslash onto parity p (Deo for p = 0, Doe for p = 1; lib/Action/fermionmatrix.cc:8-97):
//   (D in)(x) = 1/2 sum_mu [ U_mu(x) in(x+mu) - U_mu(x-mu)^dag in(x-mu) ]
// with the staggered phases folded into the links.  One thread per output site; every
// link is read exactly once per launch and shared by the NR right-hand sides the thread
// carries; neighbour spinors come through the read-only path and are reused out of L2
// (one parity of a 32^4 FP64 spinor is 25 MB, well inside the 126 MB L2).
//
// Epilogue: out = alpha*y + beta*(2 D in)/2, i.e. beta = +0.5 gives D, beta = -0.5 with
// alpha = mass^2 + sigma and y = p gives the even-even (M^dag M + sigma) p from D_oe p
// (lib/Action/Inverter/inverter.cc:206-216).  With RED the kernel also reduces, per RHS,
// Re<y, out> in FP64 (the <p, A p> of CG; each site's term formed in the spinors' precision, see
// site_dot) through reduce_finalize, whose fixed summation order makes results reproducible.
#pragma once
#include <cstring>
#include <string>

#include "autotune.h"
#include "rhmc_core.cuh"

namespace rhmc {

// Threads per block and the minimum resident blocks per SM handed to the register allocator,
// per link precision, RHS count and epilogue (RED: the solver's fused reductions, which need
// blocks of 128 or 256 threads).  A thread
// carries NR accumulators and NR neighbour spinors, so wide FP64 batches need many registers;
// the pair trades registers (spills) against resident warps (latency hiding).  The values are
// the fastest of the sweep in tune/dslash_tune.cu on B200 at 24^3x32 and 32^4; the one-RHS
// half-precision kernel, bound by instruction issue, runs fastest with the most resident warps
// (128 x 6 at 80 registers: 27.4 us at 32^4 against 31 us at 256 x 2).
template <class LF, int NR, bool RED>
struct DslashCfg {
    static constexpr bool f64 = sizeof(typename LF::real) == 8;
    static constexpr bool half1 = LF::store::planes == 1 && !f64 && NR == 1;  // H16S spinors, one RHS
    static constexpr bool narrow = (f64 && NR >= 3) || half1;
    static constexpr int block = narrow ? 128 : 256;
    static constexpr int minb = half1 ? 6 : ((f64 && NR >= 8) ? 2 : (narrow ? 3 : 2));
};

// the largest grid any configuration launches (for sizing per-block reduction partials)
constexpr int DSLASH_MIN_BLOCK = 128;

template <class LF, int NR, class FIN = NoFin>
struct DslashArgs {
    typedef typename LF::real R;
    typedef typename LF::store S;  // spinor storage of in, out, y
    typedef typename S::elem E;
    Geom g;
    int p_out;
    LF links;
    const E *in;        // NR spinors of parity 1-p_out, stride `stride` elements
    E *out;             // NR spinors of parity p_out
    const E *y;         // optional, parity p_out
    size_t stride;      // elements between consecutive RHS (>= 3*Vh)
    R alpha, beta;
    R alphas[NR];       // per-RHS alpha when use_alphas (shifted systems batched together)
    int use_alphas;
    double *partials;   // red_chunks(Vh) * NR doubles when RED
    unsigned *ticket;   // last-block counter when RED (fin() runs on the totals)
    FIN fin;
    const int *stop;    // optional: skip the launch when *stop != 0 ...
    int *stop_set;      // ... and then set *stop_set = 1 (solver loop control)
    const int *run_if;  // optional: skip the launch when *run_if == 0
    int k_lo, k_count;  // output sites [k_lo, k_lo + k_count) (k_count 0: all Vh); no RED with a range
};

// Re<y, o> of one colour added to a site's term of the fused reduction: FP64 products for FP64
// spinors; for FP32 spinors the site term is summed in FP32 with fixed rounding and converted to
// FP64 once per site and RHS (three colours' float-to-double conversions and FP64 products per
// RHS would cost more issue slots than the whole FP32 epilogue)
__device__ __forceinline__ void site_dot(double &red, float &, const cpx<double> &y, const cpx<double> &o)
{
    red += dot2(y.re, o.re, y.im, o.im);
}
__device__ __forceinline__ void site_dot(double &, float &tf, const cpx<float> &y, const cpx<float> &o)
{
    tf = __fadd_rn(tf, dot2(y.re, o.re, y.im, o.im));
}

template <class LF, int NR, bool HAS_Y, bool RED, class FIN, int BLOCK = DslashCfg<LF, NR, RED>::block,
          int MINB = DslashCfg<LF, NR, RED>::minb>
__global__ void __launch_bounds__(BLOCK, MINB) dslash_kernel(DslashArgs<LF, NR, FIN> a)
{
    typedef typename LF::real R;
    if (a.stop && *(volatile const int *)a.stop) {
        if (a.stop_set && blockIdx.x == 0 && threadIdx.x == 0) *a.stop_set = 1;
        return;
    }
    if (a.run_if && *(volatile const int *)a.run_if == 0) return;
    const int Vh = a.g.Vh;
    const int kend = a.k_count ? a.k_lo + a.k_count : Vh;
    const int ntiles = (kend - a.k_lo + BLOCK - 1) / BLOCK;
    typedef typename LF::store S;
    typedef typename S::elem E;
    // y (read only by the epilogue) is fetched into shared memory by cp.async at the start of a
    // tile, so its DRAM latency overlaps the stencil instead of following it (when it fits)
    constexpr bool PF = HAS_Y && S::soa && S::pack == 1 && (NR * S::planes * BLOCK * sizeof(E) <= 24576);
    __shared__ __align__(16) E ysm[PF ? NR * S::planes * BLOCK : 1];
    // tiles of BLOCK consecutive output sites; a launch with fewer blocks than tiles (persistent
    // blocks) walks them with stride gridDim.x, so the per-block work of the fused reduction
    // (fence, ticket) is paid once per block instead of once per tile
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int k = a.k_lo + tile * BLOCK + threadIdx.x;
        if constexpr (S::pack > 1) {
            // packed right-hand sides: one load brings P of them (PackS)
            constexpr int P = S::pack, NQ = NR / P;
            static_assert(NR % P == 0, "the batch is a whole number of packs");
            typedef PackIO<R, P> IO;
            double red[NR];
            float tf[NR];  // FP32 spinors: the site's Re<y, out>, formed in FP32 (site_dot)
#pragma unroll
            for (int j = 0; j < NR; j++) {
                red[j] = 0.0;
                tf[j] = 0.f;
            }
            if (k < kend) {
                const Site s = site_of(a.g, a.p_out, k);
                vec3<R> acc[NR];
#pragma unroll
                for (int r = 0; r < NR; r++)
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[r].c[c] = mk<R>(0, 0);
#pragma unroll
                for (int mu = 0; mu < 4; mu++) {
#pragma unroll
                    for (int dir = 0; dir < 2; dir++) {
                        su3m<R> u;
                        const int kn = neighbour(a.g, s, mu, dir ? -1 : +1);
                        if (dir == 0)
                            a.links.load(mu, a.p_out, k, u, eta_of(a.g, s, mu));
                        else
                            a.links.load(mu, 1 - a.p_out, kn, u, eta_back(a.g, s, mu));
#pragma unroll
                        for (int q = 0; q < NQ; q++) {
                            vec3<R> v[P];
#pragma unroll
                            for (int c = 0; c < 3; c++) {
                                cpx<R> e[P];
                                IO::ld(a.in + q * a.stride + (size_t)c * Vh + kn, e);
#pragma unroll
                                for (int i = 0; i < P; i++) v[i].c[c] = e[i];
                            }
#pragma unroll
                            for (int i = 0; i < P; i++) {
                                if (dir == 0)
                                    mv_acc(u, v[i], acc[q * P + i]);
                                else
                                    mdv_sub(u, v[i], acc[q * P + i]);
                            }
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < NQ; q++)
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        cpx<R> yv[P], o[P];
                        if (HAS_Y) IO::ld(a.y + q * a.stride + (size_t)c * Vh + k, yv);
#pragma unroll
                        for (int i = 0; i < P; i++) {
                            const cpx<R> A = acc[q * P + i].c[c];
                            if (HAS_Y) {
                                const R al = a.use_alphas ? a.alphas[q * P + i] : a.alpha;
                                o[i] = mk<R>(dot2(a.beta, A.re, al, yv[i].re), dot2(a.beta, A.im, al, yv[i].im));
                                if (RED) site_dot(red[q * P + i], tf[q * P + i], yv[i], o[i]);
                            } else {
                                o[i] = mk<R>(a.beta * A.re, a.beta * A.im);
                            }
                        }
                        IO::st(a.out + q * a.stride + (size_t)c * Vh + k, o);
                    }
                if (RED && sizeof(R) == 4)
#pragma unroll
                    for (int j = 0; j < NR; j++) red[j] = (double)tf[j];
            }
            if (RED) reduce_tile<NR>(red, a.partials, tile);
        } else {
            Site s = site_of(a.g, a.p_out, k < kend ? k : a.k_lo);
            if (PF && k < kend) {
#pragma unroll
                for (int r = 0; r < NR; r++)
#pragma unroll
                    for (int pl = 0; pl < S::planes; pl++)
                        cp_async_elem<sizeof(E)>(&ysm[(r * S::planes + pl) * BLOCK + threadIdx.x],
                                                 a.y + r * a.stride + (size_t)pl * Vh + k);
                cp_async_commit();
            }
            double red[NR];
            float tf[NR];
#pragma unroll
            for (int j = 0; j < NR; j++) {
                red[j] = 0.0;
                tf[j] = 0.f;
            }

            if (k < kend) {
                vec3<R> acc[NR];
#pragma unroll
                for (int r = 0; r < NR; r++)
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[r].c[c] = mk<R>(0, 0);
#pragma unroll
                for (int mu = 0; mu < 4; mu++) {
                    su3m<R> u;
                    const int kf = neighbour(a.g, s, mu, +1);
                    a.links.load(mu, a.p_out, k, u, eta_of(a.g, s, mu));
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        vec3<R> v = LF::store::template load<R>(a.in + r * a.stride, Vh, kf);
                        mv_acc(u, v, acc[r]);
                    }
                    const int kb = neighbour(a.g, s, mu, -1);
                    a.links.load(mu, 1 - a.p_out, kb, u, eta_back(a.g, s, mu));
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        vec3<R> v = LF::store::template load<R>(a.in + r * a.stride, Vh, kb);
                        mdv_sub(u, v, acc[r]);
                    }
                }
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    vec3<R> o;
                    if (HAS_Y) {
                        if (PF && r == 0) cp_async_wait_all();
                        const vec3<R> yv = PF ? S::template load_plain<R>(ysm + r * S::planes * BLOCK, BLOCK, threadIdx.x)
                                              : S::template load<R>(a.y + r * a.stride, Vh, k);
                        const R al = a.use_alphas ? a.alphas[r] : a.alpha;
#pragma unroll
                        for (int c = 0; c < 3; c++)
                            o.c[c] = mk<R>(dot2(a.beta, acc[r].c[c].re, al, yv.c[c].re),
                                           dot2(a.beta, acc[r].c[c].im, al, yv.c[c].im));
                        if (RED) {
#pragma unroll
                            for (int c = 0; c < 3; c++) site_dot(red[r], tf[r], yv.c[c], o.c[c]);
                            if (sizeof(R) == 4) red[r] = (double)tf[r];
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 3; c++) o.c[c] = mk<R>(a.beta * acc[r].c[c].re, a.beta * acc[r].c[c].im);
                    }
                    LF::store::template store<R>(a.out + r * a.stride, Vh, k, o);
                }
            }
            if (RED)
                reduce_tile<NR>(red, a.partials, tile);  // ends with a barrier
            else if (PF)
                __syncthreads();  // ysm is refilled by the next tile
        }
    }
    if (RED) reduce_last<NR>(a.partials, a.ticket, ntiles * (BLOCK / RED_CHUNK), a.fin);
}

// ------------------------------------------------------------------ launch shapes (autotune.h)
// Candidate 0 is DslashCfg's default; 1 and 2 are the two alternatives the offline sweep found
// closest for that class of instantiation (all of 128 or 256 threads, as the reductions need).
template <class LF, int NR, bool RED>
struct DsCand {
    typedef DslashCfg<LF, NR, RED> C;
    static constexpr int b0 = C::block, m0 = C::minb;
    static constexpr bool def256 = b0 == 256, def1283 = b0 == 128 && m0 == 3, def1286 = b0 == 128 && m0 == 6;
    static constexpr int b1 = def256 ? 128 : 256, m1 = def256 ? 4 : ((def1283 || def1286) ? 2 : 1);
    static constexpr int b2 = 128, m2 = def256 ? 3 : ((def1283 || def1286) ? 4 : 3);
};

// Grid of a launch over nsites output sites: one block per tile of B sites, except for the
// reducing kernels, which get one wave of persistent blocks (SMs x resident blocks) walking the
// tiles: their per-block tail (fence, ticket, barrier) is then paid once per block, which the
// sweep measured 2-9 % faster at 32^4 (FP32-12, 4 RHS: 79.5 against 85.5 us), while the plain
// kernels gain nothing from it.  The per-tile partials and their summation order do not depend
// on the grid, so both give bit-identical results.
template <class LF, int NR, bool HAS_Y, bool RED, class FIN, int B, int MB>
inline void dslash_launch_shape(const DslashArgs<LF, NR, FIN> &a, int nsites, cudaStream_t s)
{
    auto kern = dslash_kernel<LF, NR, HAS_Y, RED, FIN, B, MB>;
    const int ntiles = (nsites + B - 1) / B;
    const int grid = RED ? persistent_grid((const void *)kern, B, ntiles) : ntiles;
    kern<<<grid, B, 0, s>>>(a);
}

template <class LF, int NR, bool HAS_Y, bool RED, class FIN>
inline void dslash_launch_cand(int cand, const DslashArgs<LF, NR, FIN> &a, int nsites, cudaStream_t s)
{
    typedef DsCand<LF, NR, RED> K;
    switch (cand) {
    case 1: dslash_launch_shape<LF, NR, HAS_Y, RED, FIN, K::b1, K::m1>(a, nsites, s); break;
    case 2: dslash_launch_shape<LF, NR, HAS_Y, RED, FIN, K::b2, K::m2>(a, nsites, s); break;
    default: dslash_launch_shape<LF, NR, HAS_Y, RED, FIN, K::b0, K::m0>(a, nsites, s); break;
    }
}

template <class LF, int NR, bool HAS_Y, bool RED>
inline std::string dslash_tune_name()
{
    return std::string("dslash ") + LF::name + (LF::store::pack > 1 ? " pack=" + std::to_string(LF::store::pack) : "") +
           " nr=" + std::to_string(NR) + " y=" + std::to_string((int)HAS_Y) + " red=" + std::to_string((int)RED);
}

// Times the three candidates of an instantiation on scratch spinors (the caller's links) with
// CUDA events on stream s and records the fastest; returns its index (0 when timing fails).
template <class LF, int NR, bool HAS_Y, bool RED>
int dslash_tune(const Geom &g, const LF &links, cudaStream_t s, const std::string &key)
{
    typedef typename LF::real R;
    typedef typename LF::store::elem E;
    const size_t vec = (size_t)LF::store::planes * g.Vh;
    void *in = nullptr, *out = nullptr, *y = nullptr, *part = nullptr, *tick = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int best = 0;
    float us[3] = {0, 0, 0};
    cudaError_t e = cudaMalloc(&in, NR * vec * sizeof(E));
    if (e == cudaSuccess) e = cudaMalloc(&out, NR * vec * sizeof(E));
    if (e == cudaSuccess) e = cudaMalloc(&y, NR * vec * sizeof(E));
    if (e == cudaSuccess) e = cudaMalloc(&part, (size_t)red_chunks(g.Vh) * NR * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&tick, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(in, 0, NR * vec * sizeof(E), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(y, 0, NR * vec * sizeof(E), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(tick, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        DslashArgs<LF, NR, NoFin> t;
        memset(&t, 0, sizeof(t));
        t.g = g;
        t.p_out = 1;
        t.links = links;
        t.in = (const E *)in;
        t.out = (E *)out;
        t.y = HAS_Y ? (const E *)y : nullptr;
        t.stride = vec;
        t.alpha = (R)0.01;
        t.beta = (R)-0.5;
        t.partials = (double *)part;
        t.ticket = (unsigned *)tick;
        for (int cand = 0; cand < 3 && e == cudaSuccess; cand++) {
            dslash_launch_cand<LF, NR, HAS_Y, RED, NoFin>(cand, t, g.Vh, s);  // warm-up
            cudaEventRecord(e0, s);
            for (int r = 0; r < 4; r++) dslash_launch_cand<LF, NR, HAS_Y, RED, NoFin>(cand, t, g.Vh, s);
            cudaEventRecord(e1, s);
            e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            us[cand] = ms * 1e3f / 4.f;
        }
        if (e == cudaSuccess) {
            for (int cand = 1; cand < 3; cand++)
                if (us[cand] < us[best]) best = cand;
            typedef DsCand<LF, NR, RED> K;
            const DsShape shapes[3] = {{K::b0, K::m0}, {K::b1, K::m1}, {K::b2, K::m2}};
            tune_put(key, best, us, shapes, 3);
        }
    }
    if (e != cudaSuccess) {
        best = 0;
        cudaGetLastError();
    }
    for (void *p : {in, out, y, part, tick})
        if (p) cudaFree(p);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return best;
}

// The candidate an instantiation runs with: the override, else the tuned choice, tuning it now
// when it is unknown and the stream is not capturing, else the default.
template <class LF, int NR, bool HAS_Y, bool RED>
inline int dslash_candidate(const Geom &g, const LF &links, cudaStream_t s)
{
    if (autotune_override() >= 0) return autotune_override();
    if (!autotune_enabled()) return 0;
    const std::string key = tune_key(g.Vh, dslash_tune_name<LF, NR, HAS_Y, RED>());
    const int c = tune_get(key);
    if (c >= 0) return c;
    if (stream_capturing(s)) return 0;
    return dslash_tune<LF, NR, HAS_Y, RED>(g, links, s, key);
}

// One launch over `nsites` output sites (from a.k_lo) on stream s, in the tuned launch shape
// (code that captures launches looks the shape up with dslash_candidate before the capture).
template <class LF, int NR, bool HAS_Y, bool RED, class FIN>
inline cudaError_t dslash_launch(const DslashArgs<LF, NR, FIN> &a, int nsites, cudaStream_t s)
{
    dslash_launch_cand<LF, NR, HAS_Y, RED, FIN>(dslash_candidate<LF, NR, HAS_Y, RED>(a.g, a.links, s), a, nsites, s);
    return cudaGetLastError();
}

}  // namespace rhmc
