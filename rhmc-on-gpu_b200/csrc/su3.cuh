// su3.cuh -- FP64 SU(3) algebra for the force and update kernels.
//
// Follows the reference's Su3 class (lib/Action/su3.h, su3.cc): product, hermitian conjugate,
// traceless anti-hermitian part (Su3::ta, su3.cc:161-183), 6th-order Taylor exponential
// (Su3::exp, su3.cc:187-219) and row Gram-Schmidt unitarisation (Su3::sunitarize,
// su3.cc:69-112).  Algebra fields are stored as 8 reals per link:
//   [re a01, im a01, re a02, im a02, re a12, im a12, d0, d1]
// with, for momenta (traceless hermitian), diag = (d0, d1, -d0-d1) real, a10 = conj(a01), ...
// and, for ipdot (traceless anti-hermitian), diag = i(d0, d1, -d0-d1), a10 = -conj(a01), ...
#pragma once
#include "rhmc_core.cuh"

namespace rhmc {

typedef su3m<double> M3;
typedef cpx<double> C;

__device__ __forceinline__ M3 m3_zero()
{
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.e[i][j] = mk<double>(0, 0);
    return r;
}

__device__ __forceinline__ M3 m3_mul(const M3 &a, const M3 &b)
{
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            C s = a.e[i][0] * b.e[0][j];
            s = cmadd(a.e[i][1], b.e[1][j], s);
            s = cmadd(a.e[i][2], b.e[2][j], s);
            r.e[i][j] = s;
        }
    return r;
}

// a * b^dag
__device__ __forceinline__ M3 m3_mul_nd(const M3 &a, const M3 &b)
{
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            C s = a.e[i][0] * conj(b.e[j][0]);
            s = s + a.e[i][1] * conj(b.e[j][1]);
            s = s + a.e[i][2] * conj(b.e[j][2]);
            r.e[i][j] = s;
        }
    return r;
}

// a^dag * b
__device__ __forceinline__ M3 m3_mul_dn(const M3 &a, const M3 &b)
{
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            C s = conj(a.e[0][i]) * b.e[0][j];
            s = s + conj(a.e[1][i]) * b.e[1][j];
            s = s + conj(a.e[2][i]) * b.e[2][j];
            r.e[i][j] = s;
        }
    return r;
}

__device__ __forceinline__ void m3_add(M3 &a, const M3 &b)
{
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) a.e[i][j] = a.e[i][j] + b.e[i][j];
}

__device__ __forceinline__ void m3_scale(M3 &a, double s)
{
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) a.e[i][j] = s * a.e[i][j];
}

__device__ __forceinline__ double m3_retr(const M3 &a) { return a.e[0][0].re + a.e[1][1].re + a.e[2][2].re; }

// link U_mu at (parity p, half index k) of the FP64 master [mu][p][9][Vh] double2
__device__ __forceinline__ M3 load_link64(const double2 *__restrict__ U, int Vh, int mu, int p, int k)
{
    const double2 *b = U + (size_t)((mu * 2 + p) * 9) * Vh + k;
    M3 u;
#pragma unroll
    for (int e = 0; e < 9; e++) {
        const double2 v = __ldg(b + (size_t)e * Vh);
        u.e[e / 3][e % 3] = mk<double>(v.x, v.y);
    }
    return u;
}

__device__ __forceinline__ void store_link64(double2 *U, int Vh, int mu, int p, int k, const M3 &u)
{
    double2 *b = U + (size_t)((mu * 2 + p) * 9) * Vh + k;
#pragma unroll
    for (int e = 0; e < 9; e++) b[(size_t)e * Vh] = make_double2(u.e[e / 3][e % 3].re, u.e[e / 3][e % 3].im);
}

// traceless anti-hermitian part (Su3::ta) packed into 8 reals
__device__ __forceinline__ void ta_pack(const M3 &m, double (&o)[8])
{
    const C a01 = 0.5 * (m.e[0][1] - conj(m.e[1][0]));
    const C a02 = 0.5 * (m.e[0][2] - conj(m.e[2][0]));
    const C a12 = 0.5 * (m.e[1][2] - conj(m.e[2][1]));
    const double i0 = m.e[0][0].im, i1 = m.e[1][1].im, i2 = m.e[2][2].im;
    const double tr = (i0 + i1 + i2) * (1.0 / 3.0);
    o[0] = a01.re; o[1] = a01.im;
    o[2] = a02.re; o[3] = a02.im;
    o[4] = a12.re; o[5] = a12.im;
    o[6] = i0 - tr;
    o[7] = i1 - tr;
}

__device__ __forceinline__ void load_alg(const double *__restrict__ A, int Vh, int mu, int p, int k, double (&o)[8])
{
    const double *b = A + (size_t)((mu * 2 + p) * 8) * Vh + k;
#pragma unroll
    for (int j = 0; j < 8; j++) o[j] = b[(size_t)j * Vh];
}

__device__ __forceinline__ void store_alg(double *A, int Vh, int mu, int p, int k, const double (&o)[8])
{
    double *b = A + (size_t)((mu * 2 + p) * 8) * Vh + k;
#pragma unroll
    for (int j = 0; j < 8; j++) b[(size_t)j * Vh] = o[j];
}

// hermitian traceless matrix from its 8 reals
__device__ __forceinline__ M3 herm_unpack(const double (&a)[8])
{
    M3 m;
    m.e[0][0] = mk<double>(a[6], 0.0);
    m.e[1][1] = mk<double>(a[7], 0.0);
    m.e[2][2] = mk<double>(-a[6] - a[7], 0.0);
    m.e[0][1] = mk<double>(a[0], a[1]);
    m.e[0][2] = mk<double>(a[2], a[3]);
    m.e[1][2] = mk<double>(a[4], a[5]);
    m.e[1][0] = mk<double>(a[0], -a[1]);
    m.e[2][0] = mk<double>(a[2], -a[3]);
    m.e[2][1] = mk<double>(a[4], -a[5]);
    return m;
}

// Su3::sunitarize (row 0 normalised, row 1 Gram-Schmidt, row 2 = conj(row0 x row1)), then
// row 2 times eta (Conf::unitarize_with_eta, lib/Main/Conf/conf.cc:235-251)
__device__ __forceinline__ void sunitarize_eta(M3 &m, double eta)
{
    double n = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) n += m.e[0][i].re * m.e[0][i].re + m.e[0][i].im * m.e[0][i].im;
    n = 1.0 / sqrt(n);
#pragma unroll
    for (int i = 0; i < 3; i++) m.e[0][i] = n * m.e[0][i];
    C pr = mk<double>(0, 0);
#pragma unroll
    for (int i = 0; i < 3; i++) pr = pr + conj(m.e[0][i]) * m.e[1][i];
#pragma unroll
    for (int i = 0; i < 3; i++) m.e[1][i] = m.e[1][i] - pr * m.e[0][i];
    n = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) n += m.e[1][i].re * m.e[1][i].re + m.e[1][i].im * m.e[1][i].im;
    n = 1.0 / sqrt(n);
#pragma unroll
    for (int i = 0; i < 3; i++) m.e[1][i] = n * m.e[1][i];
    C a = m.e[0][1] * m.e[1][2] - m.e[0][2] * m.e[1][1];
    C b = m.e[0][2] * m.e[1][0] - m.e[0][0] * m.e[1][2];
    C c = m.e[0][0] * m.e[1][1] - m.e[0][1] * m.e[1][0];
    m.e[2][0] = mk<double>(eta * a.re, -eta * a.im);
    m.e[2][1] = mk<double>(eta * b.re, -eta * b.im);
    m.e[2][2] = mk<double>(eta * c.re, -eta * c.im);
}

// exp(X) by the 6th-order Taylor recursion of Su3::exp (without its final sunitarize)
__device__ __forceinline__ M3 exp_taylor6(const M3 &x)
{
    M3 r = x;
    r.e[0][0] = r.e[0][0] + mk<double>(1.0, 0.0);
    r.e[1][1] = r.e[1][1] + mk<double>(1.0, 0.0);
    r.e[2][2] = r.e[2][2] + mk<double>(1.0, 0.0);
    M3 aux = x;
    const double inv[5] = {0.5, 1.0 / 3.0, 0.25, 0.2, 1.0 / 6.0};
#pragma unroll
    for (int o = 0; o < 5; o++) {
        aux = m3_mul(aux, x);
        m3_scale(aux, inv[o]);
        m3_add(r, aux);
    }
    return r;
}

}  // namespace rhmc
