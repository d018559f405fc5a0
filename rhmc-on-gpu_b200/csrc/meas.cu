// meas.cu -- measurements on the device-resident fields:
//   polyakov_kernel  Conf::calc_poly (lib/Measurements/gaugemeas.cc:66-106): ordered product of
//                    the temporal links along each spatial point, -Tr / 3, averaged
//   chiral_kernel    the site sums of chiral_meas (lib/Measurements/chiralmeas.cc:44-183, the
//                    branch without imaginary chemical potential): chiral condensate <rnd, chi>,
//                    energy/baryon densities from the temporal hops and pressure from the
//                    spatial hops of the noise and solution fields
// rhmc_chiral_meas forms phi_e = m rnd_e - Deo rnd_o with the Dslash epilogue, solves
// (M^dag M) chi_e = phi_e with the FP64 multi-shift solver (one shift, 0), forms
// chi_o = (rnd_o - Doe chi_e) / m, and reduces.  Per-block FP64 partials are summed on the host
// in block order (deterministic).
#include <cmath>
#include <vector>

#include "capi_util.h"
#include "context.h"
#include "kernels.h"
#include "su3.cuh"

namespace rhmc {

constexpr int MEAS_BLOCK = 256;

// c_scalprod (lib/Tools/vec3.h:227-235): sum_c conj(a_c) b_c
__device__ __forceinline__ void cdot_acc(const vec3<double> &a, const vec3<double> &b, double &re, double &im)
{
#pragma unroll
    for (int c = 0; c < 3; c++) {
        re += a.c[c].re * b.c[c].re + a.c[c].im * b.c[c].im;
        im += a.c[c].re * b.c[c].im - a.c[c].im * b.c[c].re;
    }
}

__device__ __forceinline__ vec3<double> mat_vec(const M3 &u, const vec3<double> &v)
{
    vec3<double> o;
#pragma unroll
    for (int c = 0; c < 3; c++) o.c[c] = mk<double>(0.0, 0.0);
    mv_acc(u, v, o);
    return o;
}

// one thread per spatial point; the product starts where the reference's loop over its sites
// r < vol3 starts: t = 0 where x+y+z is even, t = 1 where it is odd (the even sites of the first
// two slabs), so the traces are those of the reference, not only equal up to cyclicity
__global__ void __launch_bounds__(MEAS_BLOCK) polyakov_kernel(Geom g, const double2 *__restrict__ U, double *partials)
{
    const long sp = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long vol3 = (long)g.nx * g.ny * g.nz;
    double v[2] = {0.0, 0.0};
    if (sp < vol3) {
        const int x = (int)(sp % g.nx), y = (int)((sp / g.nx) % g.ny), z = (int)(sp / ((long)g.nx * g.ny));
        int t = (x + y + z) & 1;
        M3 a;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) a.e[i][j] = mk<double>(i == j ? 1.0 : 0.0, 0.0);
        for (int n = 0; n < g.nt; n++) {
            a = m3_mul(a, load_link64(U, g.Vh, 3, (x + y + z + t) & 1, half_index(g, x, y, z, t)));
            t = (t + 1 == g.nt) ? 0 : t + 1;
        }
        v[0] = -(a.e[0][0].re + a.e[1][1].re + a.e[2][2].re);
        v[1] = -(a.e[0][0].im + a.e[1][1].im + a.e[2][2].im);
    }
    __shared__ double smem[2 * 32];
    block_sum<2>(v, smem);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = v[0];
        partials[2 * blockIdx.x + 1] = v[1];
    }
}

// thread k: even site k and odd site k (the reference's loop index i with j = i + sizeh)
__global__ void __launch_bounds__(MEAS_BLOCK) chiral_kernel(Geom g, const double2 *__restrict__ U, const double2 *__restrict__ rnd_e,
                                                           const double2 *__restrict__ rnd_o, const double2 *__restrict__ chi_e,
                                                           const double2 *__restrict__ chi_o, double *partials)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int Vh = g.Vh;
    double v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = 0.0;
    if (k < Vh) {
        const Site se = site_of(g, 0, k), so = site_of(g, 1, k);
        const vec3<double> re = load_spinor<double>(rnd_e, Vh, k), ro = load_spinor<double>(rnd_o, Vh, k);
        const vec3<double> ce = load_spinor<double>(chi_e, Vh, k), co = load_spinor<double>(chi_o, Vh, k);
        cdot_acc(ro, co, v[0], v[1]);
        cdot_acc(re, ce, v[0], v[1]);
        // temporal hops: p1 - p2 (energy) and p1 + p2 (baryon density)
        double p1r = 0, p1i = 0, p2r = 0, p2i = 0;
        {
            const M3 u = load_link64(U, Vh, 3, 0, k);
            const int kn = neighbour(g, se, 3, +1);
            cdot_acc(re, mat_vec(u, load_spinor<double>(chi_o, Vh, kn)), p1r, p1i);
            cdot_acc(mat_vec(u, load_spinor<double>(rnd_o, Vh, kn)), ce, p2r, p2i);
        }
        double q1r = 0, q1i = 0, q2r = 0, q2i = 0;
        {
            const M3 u = load_link64(U, Vh, 3, 1, k);
            const int kn = neighbour(g, so, 3, +1);
            cdot_acc(ro, mat_vec(u, load_spinor<double>(chi_e, Vh, kn)), q1r, q1i);
            cdot_acc(mat_vec(u, load_spinor<double>(rnd_e, Vh, kn)), co, q2r, q2i);
        }
        v[2] = (p1r - p2r) + (q1r - q2r);
        v[3] = (p1i - p2i) + (q1i - q2i);
        v[4] = (p1r + p2r) + (q1r + q2r);
        v[5] = (p1i + p2i) + (q1i + q2i);
        // spatial hops: pressure
#pragma unroll 1
        for (int mu = 0; mu < 3; mu++) {
            double ar = 0, ai = 0, br = 0, bi = 0;
            M3 u = load_link64(U, Vh, mu, 0, k);
            int kn = neighbour(g, se, mu, +1);
            cdot_acc(re, mat_vec(u, load_spinor<double>(chi_o, Vh, kn)), ar, ai);
            cdot_acc(mat_vec(u, load_spinor<double>(rnd_o, Vh, kn)), ce, br, bi);
            v[6] += ar - br;
            v[7] += ai - bi;
            ar = ai = br = bi = 0;
            u = load_link64(U, Vh, mu, 1, k);
            kn = neighbour(g, so, mu, +1);
            cdot_acc(ro, mat_vec(u, load_spinor<double>(chi_e, Vh, kn)), ar, ai);
            cdot_acc(mat_vec(u, load_spinor<double>(rnd_e, Vh, kn)), co, br, bi);
            v[6] += ar - br;
            v[7] += ai - bi;
        }
    }
    __shared__ double smem[8 * 32];
    block_sum<8>(v, smem);
    if (threadIdx.x == 0)
#pragma unroll
        for (int j = 0; j < 8; j++) partials[8 * (size_t)blockIdx.x + j] = v[j];
}

static int sum_partials(rhmc_ctx *c, const double *d, int nblocks, int n, double *out)
{
    std::vector<double> h((size_t)nblocks * n);
    CK(cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int j = 0; j < n; j++) out[j] = 0.0;
    for (int b = 0; b < nblocks; b++)
        for (int j = 0; j < n; j++) out[j] += h[(size_t)b * n + j];
    return RHMC_OK;
}

}  // namespace rhmc

using namespace rhmc;

extern "C" {

int rhmc_polyakov(rhmc_ctx *c, double *re, double *im)
{
    if (!c || !re || !im) return fail(RHMC_ERR_ARG, "null argument");
    const long vol3 = (long)c->g.nx * c->g.ny * c->g.nz;
    const int nb = grid_for(vol3, MEAS_BLOCK);
    void *part;
    CK(c->ws.get("meas_part", (size_t)nb * 8 * sizeof(double), &part));
    polyakov_kernel<<<nb, MEAS_BLOCK, 0, c->stream>>>(c->g, c->U64, (double *)part);
    c->launches++;
    CK(cudaGetLastError());
    double s[2] = {0.0, 0.0};
    int rc = sum_partials(c, (const double *)part, nb, 2, s);
    if (rc) return rc;
    const double inv_vol3 = 1.0 / (double)vol3, one_by_three = 1.0 / 3.0;
    *re = s[0] * inv_vol3 * one_by_three;
    *im = s[1] * inv_vol3 * one_by_three;
    return RHMC_OK;
}

int rhmc_chiral_meas(rhmc_ctx *c, int nrand, int no_flavours, const double *noise_e, const double *noise_o, double residual,
                     int max_iter, int location, double *out)
{
    if (!c || !noise_e || !noise_o || !out || nrand < 1 || max_iter < 1 || !(residual > 0.0) || c->mass <= 0.0)
        return fail(RHMC_ERR_ARG, "bad argument");
    if (location != RHMC_HOST && location != RHMC_DEVICE) return fail(RHMC_ERR_ARG, "bad location");
    const size_t n3 = 3 * (size_t)c->Vh, bytes = n3 * sizeof(double2);
    void *re, *ro, *pe, *ce, *co, *part;
    CK(c->ws.get("meas_re", bytes, &re));
    CK(c->ws.get("meas_ro", bytes, &ro));
    CK(c->ws.get("meas_pe", bytes, &pe));
    CK(c->ws.get("meas_ce", bytes, &ce));
    CK(c->ws.get("meas_co", bytes, &co));
    const int nb = grid_for(c->Vh, MEAS_BLOCK);
    CK(c->ws.get("meas_part", (size_t)nb * 8 * sizeof(double), &part));
    const double m = c->mass;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const double zero = 0.0;
    for (int r = 0; r < nrand; r++) {
        int rc = rhmc_spinor_to_internal(c, RHMC_LINKS_F64_18, re, noise_e + (size_t)r * 6 * c->Vh, 1, location);
        if (!rc) rc = rhmc_spinor_to_internal(c, RHMC_LINKS_F64_18, ro, noise_o + (size_t)r * 6 * c->Vh, 1, location);
        if (rc) return rc;
        // phi_e = m rnd_e - Deo rnd_o (chiralmeas.cc:50-55)
        CK(launch_dslash(c, RHMC_LINKS_F64_18, 0, pe, ro, n3, 1, re, m, -0.5, nullptr, nullptr));
        // (M^dag M) chi_e = phi_e (chiralmeas.cc:57-58: invert to residue_metro)
        rhmc_msolve_params mp;
        memset(&mp, 0, sizeof(mp));
        mp.nshift = 1;
        mp.shifts = &zero;
        mp.nrhs = 1;
        mp.residual = residual;
        mp.max_iter = max_iter;
        mp.mode = RHMC_MSOLVE_FP64;
        mp.fmt = RHMC_LINKS_F64_18;
        rc = rhmc_msolve(c, &mp, (double *)ce, (const double *)pe, nullptr);
        if (rc) return rc;
        // chi_o = (rnd_o - Doe chi_e) / m (chiralmeas.cc:87-91)
        CK(launch_dslash(c, RHMC_LINKS_F64_18, 1, co, ce, n3, 1, ro, 1.0 / m, -0.5 / m, nullptr, nullptr));
        chiral_kernel<<<nb, MEAS_BLOCK, 0, c->stream>>>(c->g, c->U64, (const double2 *)re, (const double2 *)ro, (const double2 *)ce,
                                                         (const double2 *)co, (double *)part);
        c->launches++;
        CK(cudaGetLastError());
        double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        rc = sum_partials(c, (const double *)part, nb, 8, s);
        if (rc) return rc;
        const double inv_size = 1.0 / (double)c->V;
        for (int j = 0; j < 8; j++) acc[j] += s[j] * ((j < 2 ? 1.0 : 0.5) * no_flavours * 0.25 * inv_size);
    }
    for (int j = 0; j < 8; j++) out[j] = acc[j] / (double)nrand;
    return RHMC_OK;
}

}  // extern "C"
