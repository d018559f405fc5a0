// force.cu -- molecular-dynamics forces on sm_100a, FP64.
//
// ipdot = TA(U (beta/3 staples + F_f)) (calc_ipdot, lib/Update/ipdot.cc:149-196).  TA is linear,
// so the gauge part and the fermion part are produced by separate kernels that either
// overwrite or add into ipdot:
//   gauge_force_kernel   TA((U beta/3) staples), staples as calc_staples (lib/Action/staples.cc:16-74)
//   fermion_force_kernel TA(U F_f) with F_f the outer products of fermionforce
//                        (lib/Action/fermionforce.cc:46-104): even x: sum a_i h_i(x+mu) (x) x_i(x)^*,
//                        odd x: -sum a_i x_i(x+mu) (x) h_i(x)^*, h_i = Doe x_i (with its 1/2).
// gauge_force_kernel runs one thread per site for a fixed mu (the block index modulo 4);
// fermion_force_kernel one thread per link, mu fastest inside a site (the four links of a site
// share the site's spinor loads through L1).  All shifted solutions of all right-hand sides are summed in registers,
// so the 18-real force matrix never goes to HBM (the reference GPU code read-modify-writes an
// 18 x 4V float buffer once per shift, lib/Cuda/cuda_fermion_force.cu:370-386).
#include <string>
#include <vector>

#include "autotune.h"
#include "capi_util.h"
#include "context.h"
#include "kernels.h"
#include "su3.cuh"

namespace rhmc {

constexpr int FORCE_BLOCK = 128;

__device__ __forceinline__ Site shifted(const Geom &g, Site s, int mu, int dir)
{
    if (mu == 0) { s.x += dir; s.x = s.x < 0 ? g.nx - 1 : (s.x >= g.nx ? 0 : s.x); }
    else if (mu == 1) { s.y += dir; s.y = s.y < 0 ? g.ny - 1 : (s.y >= g.ny ? 0 : s.y); }
    else if (mu == 2) { s.z += dir; s.z = s.z < 0 ? g.nz - 1 : (s.z >= g.nz ? 0 : s.z); }
    else { s.t += dir; s.t = s.t < 0 ? g.nt - 1 : (s.t >= g.nt ? 0 : s.t); }
    return s;
}

__device__ __forceinline__ int hidx(const Geom &g, const Site &s) { return half_index(g, s.x, s.y, s.z, s.t); }

// S_mu(x) = sum_{nu != mu} [ U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
//                          + U_nu(x+mu-nu)^dag U_mu(x-nu)^dag U_nu(x-nu) ]
// Each staple is formed row by row (one row of the two-link product live at a time), with the
// same operation order per element as a full product followed by a sum.
__device__ M3 staple_sum(const Geom &g, const double2 *__restrict__ U, int mu, int p, const Site &s)
{
    const int Vh = g.Vh, q = 1 - p;
    const Site xpm = shifted(g, s, mu, +1);
    const int kxpm = hidx(g, xpm), kx = hidx(g, s);
    M3 S = m3_zero();
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        const Site xpn = shifted(g, s, nu, +1), xmn = shifted(g, s, nu, -1), xpmmn = shifted(g, xpm, nu, -1);
        {
            // upper: (U_nu(x+mu) U_mu(x+nu)^dag) U_nu(x)^dag
            const M3 A = load_link64(U, Vh, nu, q, kxpm), B = load_link64(U, Vh, mu, q, hidx(g, xpn));
            const M3 Cm = load_link64(U, Vh, nu, p, kx);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                C t[3];
#pragma unroll
                for (int l = 0; l < 3; l++) {
                    C v = A.e[i][0] * conj(B.e[l][0]);
                    v = v + A.e[i][1] * conj(B.e[l][1]);
                    v = v + A.e[i][2] * conj(B.e[l][2]);
                    t[l] = v;
                }
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    C v = t[0] * conj(Cm.e[j][0]);
                    v = v + t[1] * conj(Cm.e[j][1]);
                    v = v + t[2] * conj(Cm.e[j][2]);
                    S.e[i][j] = S.e[i][j] + v;
                }
            }
        }
        {
            // lower: (U_mu(x-nu) U_nu(x+mu-nu))^dag U_nu(x-nu)
            const int kxmn = hidx(g, xmn);
            const M3 A = load_link64(U, Vh, mu, q, kxmn), B = load_link64(U, Vh, nu, p, hidx(g, xpmmn));
            const M3 Cm = load_link64(U, Vh, nu, q, kxmn);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                C col[3];  // column i of A B
#pragma unroll
                for (int l = 0; l < 3; l++) {
                    C v = A.e[l][0] * B.e[0][i];
                    v = cmadd(A.e[l][1], B.e[1][i], v);
                    v = cmadd(A.e[l][2], B.e[2][i], v);
                    col[l] = v;
                }
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    C v = conj(col[0]) * Cm.e[0][j];
                    v = v + conj(col[1]) * Cm.e[1][j];
                    v = v + conj(col[2]) * Cm.e[2][j];
                    S.e[i][j] = S.e[i][j] + v;
                }
            }
        }
    }
    return S;
}

// Both force kernels walk the sites in chunks of consecutive half-indices that alternate between
// the two parities (chunk c: parity c & 1, half-sites from (c >> 1) * W), so a site and its
// nearest neighbours of the other parity are handled by warps that run at about the same time.
// A link or spinor of one parity is read both by the threads of its own site and, as a
// neighbour, by the threads of the other parity: in a parity-major order those two reads lie a
// whole half-lattice apart, which at 24^4 and above is more than L2 holds, and every such
// element came from HBM twice.
constexpr int GF_CHUNK = 32;  // half-sites per warp, gauge force
constexpr int FF_CHUNK = 8;   // half-sites per warp (x 4 mu), fermion force

__host__ __device__ __forceinline__ long force_chunks(int Vh, int W) { return 2L * ((Vh + W - 1) / W); }

// mode 0: ipdot = TA(U beta/3 S); mode 1: ipdot += TA(U beta/3 S).
// One thread per site for one mu: a warp covers 32 consecutive half-sites of one parity, so every
// link-plane load of the warp is one contiguous 512-byte segment (own links) or nearly so
// (neighbour links).  mu is the fastest-varying block index, so the four blocks of a site range
// run together and share their links through L2 (with mu as the slow index the whole link field
// was streamed from HBM once per mu).  At 3 resident blocks per SM the register budget is 170
// per thread with no spills.
__global__ void __launch_bounds__(FORCE_BLOCK, 3) gauge_force_kernel(Geom g, const double2 *__restrict__ U, double *IP,
                                                                      double beta_by_three, int mode)
{
    const int mu = blockIdx.x & 3;
    const int Vh = g.Vh;
    const long chunk = (long)(blockIdx.x >> 2) * (FORCE_BLOCK / 32) + (threadIdx.x >> 5);
    if (chunk >= force_chunks(Vh, GF_CHUNK)) return;
    const int p = (int)(chunk & 1);
    const int k = (int)(chunk >> 1) * GF_CHUNK + (threadIdx.x & 31);
    if (k >= Vh) return;
    const Site s = site_of(g, p, k);
    const M3 S = staple_sum(g, U, mu, p, s);
    M3 us = m3_mul(load_link64(U, Vh, mu, p, k), S);
    m3_scale(us, beta_by_three);
    double o[8];
    ta_pack(us, o);
    if (mode) {
        double c[8];
        load_alg(IP, Vh, mu, p, k, c);
#pragma unroll
        for (int j = 0; j < 8; j++) o[j] += c[j];
    }
    store_alg(IP, Vh, mu, p, k, o);
}

// x: even FP64 spinors [nv], h = Doe x: odd FP64 spinors [nv]; coef[v] the numerator of vector v.
// UNR vectors are unrolled (their loads issued together) and MINB blocks are kept resident per
// SM; the kernel waits on its loads more than on its FMAs, so the pair that keeps most bytes in
// flight wins, and the autotuner picks it per volume and vector count (FF_SHAPES).
template <int UNR, int MINB>
__global__ void __launch_bounds__(FORCE_BLOCK, MINB) fermion_force_kernel(Geom g, const double2 *__restrict__ U,
                                                                           const double2 *__restrict__ x,
                                                                           const double2 *__restrict__ h, int nv,
                                                                           const double *__restrict__ coef, double *IP,
                                                                           int mode)
{
    // a warp: FF_CHUNK half-sites of one parity x 4 mu, mu the fastest thread index
    const int Vh = g.Vh;
    const long chunk = (long)blockIdx.x * (FORCE_BLOCK / 32) + (threadIdx.x >> 5);
    if (chunk >= force_chunks(Vh, FF_CHUNK)) return;
    const int mu = threadIdx.x & 3;
    const int p = (int)(chunk & 1);
    const int k = (int)(chunk >> 1) * FF_CHUNK + ((threadIdx.x & 31) >> 2);
    if (k >= Vh) return;
    const Site s = site_of(g, p, k);
    const int kn = neighbour(g, s, mu, +1);  // x+mu, opposite parity
    const size_t stride = 3 * (size_t)Vh;
    // even x: a h(x+mu) (x) x(x)^* ; odd x: -a x(x+mu) (x) h(x)^*
    const double2 *left = p == 0 ? h : x;
    const double2 *right = p == 0 ? x : h;
    const int kl = kn, kr = k;
    const double sgn = p == 0 ? 1.0 : -1.0;
    M3 F = m3_zero();
#pragma unroll UNR
    for (int v = 0; v < nv; v++) {
        const double a = sgn * __ldg(coef + v);
        const double2 *L = left + v * stride, *R = right + v * stride;
        C l[3], r[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double2 lv = __ldg(L + (size_t)c * Vh + kl), rv = __ldg(R + (size_t)c * Vh + kr);
            l[c] = mk<double>(a * lv.x, a * lv.y);
            r[c] = mk<double>(rv.x, -rv.y);
        }
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) F.e[i][j] = cmadd(l[i], r[j], F.e[i][j]);
    }
    const M3 uf = m3_mul(load_link64(U, Vh, mu, p, k), F);
    double o[8];
    ta_pack(uf, o);
    if (mode) {
        double c[8];
        load_alg(IP, Vh, mu, p, k, c);
#pragma unroll
        for (int j = 0; j < 8; j++) o[j] += c[j];
    }
    store_alg(IP, Vh, mu, p, k, o);
}

int gauge_force(rhmc_ctx *c, int mode)
{
    const long grid = 4L * grid_for(force_chunks(c->Vh, GF_CHUNK), FORCE_BLOCK / 32);
    gauge_force_kernel<<<(unsigned)grid, FORCE_BLOCK, 0, c->stream>>>(c->g, c->U64, c->IP, c->beta / 3.0, mode);
    c->launches++;
    CK(cudaGetLastError());
    return RHMC_OK;
}

// (vectors unrolled, minimum resident blocks per SM) of the fermion force's launch candidates;
// candidate 0 is the default when tuning is off
constexpr int FF_NCAND = 4;
constexpr int FF_SHAPES[FF_NCAND][2] = {{2, 1}, {4, 1}, {2, 6}, {4, 4}};

static void ff_launch(int cand, const rhmc_ctx *c, const double2 *x, const double2 *h, int nv, const double *co,
                      double *IP, int mode)
{
    const unsigned grid = (unsigned)grid_for(force_chunks(c->Vh, FF_CHUNK), FORCE_BLOCK / 32);
    switch (cand) {
    case 1: fermion_force_kernel<4, 1><<<grid, FORCE_BLOCK, 0, c->stream>>>(c->g, c->U64, x, h, nv, co, IP, mode); break;
    case 2: fermion_force_kernel<2, 6><<<grid, FORCE_BLOCK, 0, c->stream>>>(c->g, c->U64, x, h, nv, co, IP, mode); break;
    case 3: fermion_force_kernel<4, 4><<<grid, FORCE_BLOCK, 0, c->stream>>>(c->g, c->U64, x, h, nv, co, IP, mode); break;
    default: fermion_force_kernel<2, 1><<<grid, FORCE_BLOCK, 0, c->stream>>>(c->g, c->U64, x, h, nv, co, IP, mode); break;
    }
}

// The candidate for nv vectors at this volume: the override, the recorded choice, or (first call,
// stream not capturing) the fastest of the candidates timed with CUDA events into a scratch
// ipdot (mode 0, so the context's ipdot is untouched), else 0.
static int ff_candidate(rhmc_ctx *c, const double2 *x, const double2 *h, int nv, const double *co)
{
    if (autotune_override() >= 0) return autotune_override() < FF_NCAND ? autotune_override() : 0;
    if (!autotune_enabled()) return 0;
    const std::string key = tune_key(c->Vh, "fermion_force nv=" + std::to_string(nv));
    const int got = tune_get(key);
    if (got >= 0) return got;
    if (stream_capturing(c->stream)) return 0;
    double *ip = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float us[FF_NCAND] = {0, 0, 0, 0};
    int best = 0;
    cudaError_t e = cudaMalloc(&ip, 8 * 8 * (size_t)c->Vh * sizeof(double));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    for (int k = 0; k < FF_NCAND && e == cudaSuccess; k++) {
        ff_launch(k, c, x, h, nv, co, ip, 0);  // warm-up
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 3; r++) ff_launch(k, c, x, h, nv, co, ip, 0);
        cudaEventRecord(e1, c->stream);
        e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        us[k] = ms * 1e3f / 3.f;
    }
    if (e == cudaSuccess) {
        for (int k = 1; k < FF_NCAND; k++)
            if (us[k] < us[best]) best = k;
        DsShape shapes[FF_NCAND];
        for (int k = 0; k < FF_NCAND; k++) shapes[k] = DsShape{FORCE_BLOCK, FF_SHAPES[k][1]};
        tune_put(key, best, us, shapes, FF_NCAND);
    } else {
        best = 0;
        cudaGetLastError();
    }
    if (ip) cudaFree(ip);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return best;
}

// x: [nrhs][nshift] FP64 internal even spinors; a: numerators per shift
int fermion_force(rhmc_ctx *c, int nrhs, int nshift, const double *a, const double2 *x, int mode)
{
    const int nv = nrhs * nshift;
    const size_t stride = 3 * (size_t)c->Vh;
    void *h, *co;
    CK(c->ws.get("ff_h", (size_t)nv * stride * sizeof(double2), &h));
    CK(c->ws.get("ff_coef", (size_t)nv * sizeof(double), &co));
    std::vector<double> hc(nv);
    for (int v = 0; v < nv; v++) hc[v] = a[v % nshift];
    CK(cudaMemcpyAsync(co, hc.data(), nv * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    // h = Doe x for every vector, links read once per batch of up to 8
    cudaError_t e = launch_dslash(c, RHMC_LINKS_F64_18, 1, h, x, stride, nv, nullptr, 0.0, 0.5, nullptr, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "fermion_force dslash");
    const int cand = ff_candidate(c, x, (const double2 *)h, nv, (const double *)co);
    ff_launch(cand, c, x, (const double2 *)h, nv, (const double *)co, c->IP, mode);
    c->launches++;
    CK(cudaGetLastError());
    return RHMC_OK;
}

}  // namespace rhmc

using namespace rhmc;

extern "C" {

int rhmc_gauge_force(rhmc_ctx *c, int add)
{
    if (!c) return fail(RHMC_ERR_ARG, "null context");
    return gauge_force(c, add ? 1 : 0);
}

int rhmc_fermion_force(rhmc_ctx *c, int nrhs, int nshift, const double *numerators, const double *x, int add)
{
    if (!c || !numerators || !x || nrhs < 1 || nshift < 1) return fail(RHMC_ERR_ARG, "bad argument");
    return fermion_force(c, nrhs, nshift, numerators, (const double2 *)x, add ? 1 : 0);
}

}  // extern "C"
