// update.cu -- momentum and link updates, actions and the plaquette (FP64).
//
//   mom_update_kernel   P += i step ipdot            (momenta_sum_multiply, lib/Update/momenta.cc:82-115)
//   link_update_kernel  U <- exp(i step P) U, then unitarised with eta
//                       (conf_left_exp_multiply, momenta.cc:42-78; Su3::exp, su3.cc:187-219;
//                        Conf::unitarize_with_eta, lib/Main/Conf/conf.cc:235-251)
//   plaq_kernel         per-site sums of ReTr(plaquette) split temporal/spatial, for the gauge
//                       action (Conf::loc_action, lib/Action/action.cc:6-61) and the plaquette
//                       (Conf::calc_plaq, lib/Measurements/gaugemeas.cc:7-65)
//   mom_action_kernel   sum 1/2 Tr P^2                (calc_action, action.cc:122-134)
//   rdot_kernel         Re<a, b> over one parity      (fermion_action, action.cc:65-107)
//   rational_sum_kernel out = a0 b + sum_i a_i x_i    (rationalapprox.cc:300-311; cuda_sol_sum.cu:168-221)
// Reductions write per-block FP64 partials that the host sums in block order (deterministic).
#include <vector>

#include "capi_util.h"
#include "context.h"
#include "kernels.h"
#include "su3.cuh"

namespace rhmc {

constexpr int UPD_BLOCK = 256;

__global__ void __launch_bounds__(UPD_BLOCK) mom_update_planes(int Vh, double *P, const double *__restrict__ IP, double step)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 8L * Vh) return;
    const long mp = i / Vh, k = i % Vh;
    double *p = P + mp * 8 * Vh + k;
    const double *a = IP + mp * 8 * Vh + k;
    // off-diagonal: (i step)(re + i im) = -step im + i step re
#pragma unroll
    for (int e = 0; e < 3; e++) {
        const double re = a[(2 * e) * (size_t)Vh], im = a[(2 * e + 1) * (size_t)Vh];
        p[(2 * e) * (size_t)Vh] += -step * im;
        p[(2 * e + 1) * (size_t)Vh] += step * re;
    }
    // diagonal: (i step)(i d) = -step d
    p[6 * (size_t)Vh] += -step * a[6 * (size_t)Vh];
    p[7 * (size_t)Vh] += -step * a[7 * (size_t)Vh];
}

__global__ void __launch_bounds__(UPD_BLOCK) link_update_kernel(Geom g, double2 *U, const double *__restrict__ P, double step)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int Vh = g.Vh;
    if (i >= 8L * Vh) return;
    const int mp = (int)(i / Vh), k = (int)(i % Vh);
    const int mu = mp >> 1, p = mp & 1;
    double a[8];
    load_alg(P, Vh, mu, p, k, a);
    M3 h = herm_unpack(a);
    // X = i step P
    M3 x;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) x.e[r][c] = mk<double>(-step * h.e[r][c].im, step * h.e[r][c].re);
    M3 e = exp_taylor6(x);
    sunitarize_eta(e, 1.0);  // Su3::exp ends with sunitarize
    M3 u = m3_mul(e, load_link64(U, Vh, mu, p, k));
    const Site s = site_of(g, p, k);
    sunitarize_eta(u, (double)eta_of(g, s, mu));
    store_link64(U, Vh, mu, p, k, u);
}

// temporal and spatial sums of ReTr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag): one thread per
// site (both parities) and pair of planes, {(0,1),(2,3)}, {(0,2),(1,3)} or {(0,3),(1,2)} (two
// plaquettes each, every link direction used twice), with the pair as the fastest block index
// so that the three threads of a site range run together and share its links in L2.
__global__ void __launch_bounds__(UPD_BLOCK) plaq_kernel(Geom g, const double2 *__restrict__ U, double *partials)
{
    const int pair = blockIdx.x % 3;
    const long t = (long)(blockIdx.x / 3) * blockDim.x + threadIdx.x;
    const int Vh = g.Vh;
    double v[2] = {0.0, 0.0};
    if (t < 2L * Vh) {
        const int p = t >= Vh, q = 1 - p;
        const int k = (int)(t - (long)p * Vh);
        const Site s = site_of(g, p, k);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int mu = h == 0 ? 0 : (pair == 0 ? 2 : 1);
            const int nu = h == 0 ? pair + 1 : (pair == 2 ? 2 : 3);
            M3 a = m3_mul(load_link64(U, Vh, mu, p, k), load_link64(U, Vh, nu, q, neighbour(g, s, mu, +1)));
            a = m3_mul_nd(a, load_link64(U, Vh, mu, q, neighbour(g, s, nu, +1)));
            a = m3_mul_nd(a, load_link64(U, Vh, nu, p, k));
            v[nu == 3 ? 0 : 1] += m3_retr(a);
        }
    }
    __shared__ double smem[2 * 32];
    block_sum<2>(v, smem);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = v[0];
        partials[2 * blockIdx.x + 1] = v[1];
    }
}

__global__ void __launch_bounds__(UPD_BLOCK) mom_action_kernel(int Vh, const double *__restrict__ P, double *partials)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (i < 8L * Vh) {
        const long mp = i / Vh, k = i % Vh;
        const double *a = P + mp * 8 * Vh + k;
        double off = 0.0;
#pragma unroll
        for (int j = 0; j < 6; j++) off += a[j * (size_t)Vh] * a[j * (size_t)Vh];
        const double d0 = a[6 * (size_t)Vh], d1 = a[7 * (size_t)Vh], d2 = -d0 - d1;
        v[0] = 0.5 * (d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * off);
    }
    __shared__ double smem[32];
    block_sum<1>(v, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

__global__ void __launch_bounds__(UPD_BLOCK) rdot_kernel(long n, const double2 *__restrict__ a, const double2 *__restrict__ b,
                                                         double *partials)
{
    double v[1] = {0.0};
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double2 x = a[i], y = b[i];
        v[0] += x.x * y.x + x.y * y.y;
    }
    __shared__ double smem[32];
    block_sum<1>(v, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// out[r] = a0 b[r] + sum_i a_i x[r][i]   (all FP64 internal, even)
// add: out += a0 b + sum_i a_i x_i (a rational sum accumulated over groups of poles)
__global__ void __launch_bounds__(UPD_BLOCK) rational_sum_kernel(long nel, int nrhs, int nshift, double a0,
                                                                 const double *__restrict__ a, const double2 *__restrict__ x,
                                                                 const double2 *__restrict__ b, double2 *out, int add)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // over nrhs * nel
    if (i >= (long)nrhs * nel) return;
    const long r = i / nel, e = i % nel;
    const double2 bv = b[i];
    double re = a0 * bv.x, im = a0 * bv.y;
    if (add) {
        const double2 ov = out[i];
        re += ov.x;
        im += ov.y;
    }
    for (int s = 0; s < nshift; s++) {
        const double2 xv = x[(r * nshift + s) * nel + e];
        re += __ldg(a + s) * xv.x;
        im += __ldg(a + s) * xv.y;
    }
    out[i] = make_double2(re, im);
}

static int host_sum(rhmc_ctx *c, const double *dpart, int nblocks, int n, double *out)
{
    std::vector<double> h((size_t)nblocks * n);
    CK(cudaMemcpyAsync(h.data(), dpart, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int j = 0; j < n; j++) out[j] = 0.0;
    for (int b = 0; b < nblocks; b++)
        for (int j = 0; j < n; j++) out[j] += h[(size_t)b * n + j];
    return RHMC_OK;
}

int mom_update(rhmc_ctx *c, double step)
{
    mom_update_planes<<<grid_for(8L * c->Vh, UPD_BLOCK), UPD_BLOCK, 0, c->stream>>>((int)c->Vh, c->P, c->IP, step);
    c->launches++;
    CK(cudaGetLastError());
    return RHMC_OK;
}

int link_update(rhmc_ctx *c, double step)
{
    link_update_kernel<<<grid_for(8L * c->Vh, UPD_BLOCK), UPD_BLOCK, 0, c->stream>>>(c->g, c->U64, c->P, step);
    c->launches++;
    invalidate_links(c);
    CK(cudaGetLastError());
    return RHMC_OK;
}

// sums over all sites of ReTr(plaquette): temporal (nu = 3) and spatial
int plaquette_sums(rhmc_ctx *c, double *temporal, double *spatial)
{
    const int nb = 3 * grid_for(2L * c->Vh, UPD_BLOCK);  // 3 pairs of planes per site range
    void *part;
    CK(c->ws.get("red_part", (size_t)nb * 2 * sizeof(double), &part));
    plaq_kernel<<<nb, UPD_BLOCK, 0, c->stream>>>(c->g, c->U64, (double *)part);
    c->launches++;
    CK(cudaGetLastError());
    double o[2] = {0.0, 0.0};
    int rc = host_sum(c, (const double *)part, nb, 2, o);
    *temporal = o[0];
    *spatial = o[1];
    return rc;
}

int momentum_action(rhmc_ctx *c, double *out)
{
    const int nb = grid_for(8L * c->Vh, UPD_BLOCK);
    void *part;
    CK(c->ws.get("red_part", (size_t)nb * 2 * sizeof(double), &part));
    mom_action_kernel<<<nb, UPD_BLOCK, 0, c->stream>>>((int)c->Vh, c->P, (double *)part);
    c->launches++;
    CK(cudaGetLastError());
    return host_sum(c, (const double *)part, nb, 1, out);
}

int rdot(rhmc_ctx *c, const double2 *a, const double2 *b, long n, double *out)
{
    const int nb = 148 * 4;
    void *part;
    CK(c->ws.get("red_part2", (size_t)nb * sizeof(double), &part));
    rdot_kernel<<<nb, UPD_BLOCK, 0, c->stream>>>(n, a, b, (double *)part);
    c->launches++;
    CK(cudaGetLastError());
    return host_sum(c, (const double *)part, nb, 1, out);
}

int rational_sum(rhmc_ctx *c, int nrhs, int nshift, double a0, const double *a, const double2 *x, const double2 *b, double2 *out,
                 int add)
{
    const long nel = 3 * c->Vh;
    void *da;
    CK(c->ws.get("rs_coef", (size_t)nshift * sizeof(double), &da));
    CK(cudaMemcpyAsync(da, a, nshift * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    rational_sum_kernel<<<grid_for(nrhs * nel, UPD_BLOCK), UPD_BLOCK, 0, c->stream>>>(nel, nrhs, nshift, a0, (const double *)da, x,
                                                                                      b, out, add);
    c->launches++;
    CK(cudaGetLastError());
    return RHMC_OK;
}

}  // namespace rhmc

using namespace rhmc;

extern "C" {

int rhmc_mom_update(rhmc_ctx *c, double step)
{
    if (!c) return fail(RHMC_ERR_ARG, "null context");
    return mom_update(c, step);
}

int rhmc_link_update(rhmc_ctx *c, double step)
{
    if (!c) return fail(RHMC_ERR_ARG, "null context");
    return link_update(c, step);
}

int rhmc_gauge_action(rhmc_ctx *c, double *out)
{
    if (!c || !out) return fail(RHMC_ERR_ARG, "bad argument");
    double t, s;
    int rc = plaquette_sums(c, &t, &s);
    if (rc) return rc;
    *out = (c->beta / 3.0) * (t + s);
    return RHMC_OK;
}

int rhmc_plaquette(rhmc_ctx *c, double *spatial, double *temporal)
{
    if (!c || !spatial || !temporal) return fail(RHMC_ERR_ARG, "bad argument");
    double t, s;
    int rc = plaquette_sums(c, &t, &s);
    if (rc) return rc;
    // minus sign for the phases folded into the links; 3 planes per site and 3 colours
    const double norm = 1.0 / (9.0 * (double)c->V);
    *temporal = -t * norm;
    *spatial = -s * norm;
    return RHMC_OK;
}

int rhmc_momentum_action(rhmc_ctx *c, double *out)
{
    if (!c || !out) return fail(RHMC_ERR_ARG, "bad argument");
    return momentum_action(c, out);
}

int rhmc_rdot(rhmc_ctx *c, const double *a, const double *b, int n, double *out)
{
    if (!c || !a || !b || !out || n < 1) return fail(RHMC_ERR_ARG, "bad argument");
    return rdot(c, (const double2 *)a, (const double2 *)b, (long)n * 3 * c->Vh, out);
}

int rhmc_rational_sum(rhmc_ctx *c, int nrhs, int nshift, double a0, const double *a, const double *x, const double *b, double *out)
{
    if (!c || !a || !x || !b || !out || nrhs < 1 || nshift < 0) return fail(RHMC_ERR_ARG, "bad argument");
    return rational_sum(c, nrhs, nshift, a0, a, (const double2 *)x, (const double2 *)b, (double2 *)out, 0);
}

}  // extern "C"
