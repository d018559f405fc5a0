// rhmc_core.cuh -- device-side building blocks shared by every kernel of librhmc_b200.
//
// Lattice: even/odd ordering of coppolachan/RHMC-on-GPU (lib/Main/Geometry/geometry.cc:5-11,86):
// site (parity p, half index k) has lex = x + nx*(y + ny*(z + nz*t)) with k = lex/2.
// Neighbours and staggered phases are computed from coordinates in the kernels instead of
// being read from int tables (saves 32 B/site of HBM traffic per half-Dslash); the table
// kernel in lattice.cu uses the same functions, so its bit-exact comparison with the
// reference's make_shift_table (lib/Tools/Packer/packer.cc:415-439) covers the Dslash too.
//
// Field layouts in HBM (structure of arrays, one plane per complex element so that a warp
// reads 32 consecutive sites per load instruction):
//   links    [mu][parity][plane][Vh]  (planes per format below)
//   spinor   [colour][Vh]             complex (double2 or float2); R right-hand sides are
//                                      consecutive spinors (stride 3*Vh elements)
//   algebra  [mu][parity][8][Vh]      reals: traceless (anti-)hermitian matrices
#pragma once
#include <cfloat>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace rhmc {

// ------------------------------------------------------------------ complex helpers
template <typename R> struct cpx;
template <> struct cpx<double> { double re, im; };
template <> struct cpx<float> { float re, im; };

template <typename R> __host__ __device__ __forceinline__ cpx<R> mk(R a, R b) { cpx<R> c; c.re = a; c.im = b; return c; }
template <typename R> __device__ __forceinline__ cpx<R> operator+(cpx<R> a, cpx<R> b) { return mk<R>(a.re + b.re, a.im + b.im); }
template <typename R> __device__ __forceinline__ cpx<R> operator-(cpx<R> a, cpx<R> b) { return mk<R>(a.re - b.re, a.im - b.im); }
template <typename R> __device__ __forceinline__ cpx<R> operator*(cpx<R> a, cpx<R> b) { return mk<R>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
template <typename R> __device__ __forceinline__ cpx<R> operator*(R s, cpx<R> a) { return mk<R>(s * a.re, s * a.im); }
template <typename R> __device__ __forceinline__ cpx<R> conj(cpx<R> a) { return mk<R>(a.re, -a.im); }
// a*b + c, a^* b + c
template <typename R> __device__ __forceinline__ cpx<R> cmadd(cpx<R> a, cpx<R> b, cpx<R> c)
{ return mk<R>(c.re + a.re * b.re - a.im * b.im, c.im + a.re * b.im + a.im * b.re); }
template <typename R> __device__ __forceinline__ cpx<R> cjmadd(cpx<R> a, cpx<R> b, cpx<R> c)
{ return mk<R>(c.re + a.re * b.re + a.im * b.im, c.im + a.re * b.im - a.im * b.re); }

template <typename R> struct su3m { cpx<R> e[3][3]; };
template <typename R> struct vec3 { cpx<R> c[3]; };

// ------------------------------------------------------------------ lattice geometry
// n / d for 0 <= n < 2^31 and d >= 2 as a multiply-high and a shift: with l = ceil(log2 d) and
// m = ceil(2^(31+l) / d) (< 2^32), m d - 2^(31+l) < d <= 2^l, which keeps n m / 2^(31+l) within
// the same integer as n / d for every n < 2^31 (the round-up method of Granlund and Montgomery,
// "Division by invariant integers using multiplication", 1994).  A runtime integer division
// compiles to some twenty instructions; site_of needs three per site.
struct FastDiv {
    unsigned m;
    int s;  // l - 1
};
inline FastDiv make_fastdiv(unsigned d)
{
    int l = 0;
    while ((1u << l) < d) l++;
    FastDiv f;
    f.m = (unsigned)((((unsigned long long)1 << (31 + l)) + d - 1) / d);
    f.s = l - 1;
    return f;
}
__host__ __device__ __forceinline__ unsigned fdiv(unsigned n, FastDiv f)
{
#ifdef __CUDA_ARCH__
    return __umulhi(n, f.m) >> f.s;
#else
    return (unsigned)(((unsigned long long)n * f.m) >> 32) >> f.s;
#endif
}

struct Geom {
    int nx, ny, nz, nt;
    int Vh;          // sites per parity
    int antiperiodic_t;  // 1: fermion phases flip on t = nt-1 (ferm_temp_bc == 0)
    FastDiv dx, dy, dz;  // divisions by nx, ny, nz (set by geom_divisors)
};

// fills the divisors of g from its extents (every extent is even, hence >= 2)
inline void geom_divisors(Geom &g)
{
    g.dx = make_fastdiv((unsigned)g.nx);
    g.dy = make_fastdiv((unsigned)g.ny);
    g.dz = make_fastdiv((unsigned)g.nz);
}

struct Site { int x, y, z, t; };

// coordinates of (parity p, half index k)
__host__ __device__ __forceinline__ Site site_of(const Geom &g, int p, int k)
{
    const unsigned lex2 = 2u * (unsigned)k;
    unsigned r = fdiv(lex2, g.dx);
    const int x0 = (int)(lex2 - r * (unsigned)g.nx);
    Site s;
    unsigned q = fdiv(r, g.dy);
    s.y = (int)(r - q * (unsigned)g.ny);
    r = q;
    q = fdiv(r, g.dz);
    s.z = (int)(r - q * (unsigned)g.nz);
    s.t = (int)q;
    s.x = x0 + ((p + x0 + s.y + s.z + s.t) & 1);
    return s;
}

__host__ __device__ __forceinline__ int half_index(const Geom &g, int x, int y, int z, int t)
{
    return (x + g.nx * (y + g.ny * (z + g.nz * t))) >> 1;
}

// half index of the neighbour x + dir*mu (dir = +1/-1), periodic in every direction
__host__ __device__ __forceinline__ int neighbour(const Geom &g, Site s, int mu, int dir)
{
    int x = s.x, y = s.y, z = s.z, t = s.t;
    if (mu == 0) { x += dir; x = (x < 0) ? g.nx - 1 : (x >= g.nx ? 0 : x); }
    else if (mu == 1) { y += dir; y = (y < 0) ? g.ny - 1 : (y >= g.ny ? 0 : y); }
    else if (mu == 2) { z += dir; z = (z < 0) ? g.nz - 1 : (z >= g.nz ? 0 : z); }
    else { t += dir; t = (t < 0) ? g.nt - 1 : (t >= g.nt ? 0 : t); }
    return half_index(g, x, y, z, t);
}

// staggered phase eta_mu(x) (geometry.cc:107-153) with the antiperiodic time boundary
__host__ __device__ __forceinline__ int eta_of(const Geom &g, Site s, int mu)
{
    int e;
    if (mu == 0) e = 1;
    else if (mu == 1) e = 1 - 2 * (s.x & 1);
    else if (mu == 2) e = 1 - 2 * ((s.x + s.y) & 1);
    else {
        e = 1 - 2 * ((s.x + s.y + s.z) & 1);
        if (g.antiperiodic_t && s.t == g.nt - 1) e = -e;
    }
    return e;
}

// eta of the link U_mu(x - mu): equal to eta_mu(x) except for the time boundary flip
__host__ __device__ __forceinline__ int eta_back(const Geom &g, Site s, int mu)
{
    int e;
    if (mu == 0) e = 1;
    else if (mu == 1) e = 1 - 2 * (s.x & 1);
    else if (mu == 2) e = 1 - 2 * ((s.x + s.y) & 1);
    else {
        e = 1 - 2 * ((s.x + s.y + s.z) & 1);
        if (g.antiperiodic_t && s.t == 0) e = -e;
    }
    return e;
}

// ------------------------------------------------------------------ link formats
// Row 2 is reconstructed as eta * conj(row0 x row1), the relation Conf::unitarize_with_eta
// (lib/Main/Conf/conf.cc:235-251) leaves in every stored link; the reference GPU code
// reconstructs the same way (lib/Cuda/cuda_rhmc.cuh:32-45).
template <typename R>
__device__ __forceinline__ void reconstruct_row2(su3m<R> &u, R eta)
{
    cpx<R> a = u.e[0][1] * u.e[1][2] - u.e[0][2] * u.e[1][1];
    cpx<R> b = u.e[0][2] * u.e[1][0] - u.e[0][0] * u.e[1][2];
    cpx<R> c = u.e[0][0] * u.e[1][1] - u.e[0][1] * u.e[1][0];
    u.e[2][0] = mk<R>(eta * a.re, -eta * a.im);
    u.e[2][1] = mk<R>(eta * b.re, -eta * b.im);
    u.e[2][2] = mk<R>(eta * c.re, -eta * c.im);
}

// Spinor storage policies (defined below): every link format names the storage of the spinors
// its Dslash reads and writes.
struct F64S;
struct F32S;
struct H16S;
struct A64S;

// FP64, 18 reals: 9 double2 planes
struct L64_18 {
    typedef double real;
    typedef F64S store;
    static constexpr const char *name = "f64_18";
    static constexpr int planes = 9;
    static constexpr int reals = 18;
    static constexpr int bytes = 144;
    const double2 *__restrict__ p;
    int Vh;
    __device__ __forceinline__ void load(int mu, int par, int k, su3m<double> &u, int) const
    {
        const double2 *b = p + (size_t)((mu * 2 + par) * 9) * Vh + k;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            double2 v = __ldg(b + (size_t)e * Vh);
            u.e[e / 3][e % 3] = mk<double>(v.x, v.y);
        }
    }
};

// FP64 18-real links with spinors in the reference's site-major host layout (A64S)
struct L64_18A : L64_18 {
    typedef A64S store;
    static constexpr const char *name = "f64_18_host";
};

// FP64, 12 reals: 6 double2 planes, row 2 reconstructed
struct L64_12 {
    typedef double real;
    typedef F64S store;
    static constexpr const char *name = "f64_12";
    static constexpr int planes = 6;
    static constexpr int reals = 12;
    static constexpr int bytes = 96;
    const double2 *__restrict__ p;
    int Vh;
    __device__ __forceinline__ void load(int mu, int par, int k, su3m<double> &u, int eta) const
    {
        const double2 *b = p + (size_t)((mu * 2 + par) * 6) * Vh + k;
#pragma unroll
        for (int e = 0; e < 6; e++) {
            double2 v = __ldg(b + (size_t)e * Vh);
            u.e[e / 3][e % 3] = mk<double>(v.x, v.y);
        }
        reconstruct_row2<double>(u, (double)eta);
    }
};

// FP32, 18 reals: 4 float4 planes + 1 float2 plane (the float2 planes follow all float4 ones)
struct L32_18 {
    typedef float real;
    typedef F32S store;
    static constexpr const char *name = "f32_18";
    static constexpr int planes = 5;
    static constexpr int reals = 18;
    static constexpr int bytes = 72;
    const float4 *__restrict__ p;
    int Vh;
    __device__ __forceinline__ void load(int mu, int par, int k, su3m<float> &u, int) const
    {
        const float4 *b = p + (size_t)((mu * 2 + par) * 4) * Vh + k;
        float4 a0 = __ldg(b), a1 = __ldg(b + Vh), a2 = __ldg(b + 2 * (size_t)Vh), a3 = __ldg(b + 3 * (size_t)Vh);
        const float2 *q = reinterpret_cast<const float2 *>(p + (size_t)32 * Vh) + (size_t)(mu * 2 + par) * Vh + k;
        float2 a4 = __ldg(q);
        u.e[0][0] = mk<float>(a0.x, a0.y); u.e[0][1] = mk<float>(a0.z, a0.w);
        u.e[0][2] = mk<float>(a1.x, a1.y); u.e[1][0] = mk<float>(a1.z, a1.w);
        u.e[1][1] = mk<float>(a2.x, a2.y); u.e[1][2] = mk<float>(a2.z, a2.w);
        u.e[2][0] = mk<float>(a3.x, a3.y); u.e[2][1] = mk<float>(a3.z, a3.w);
        u.e[2][2] = mk<float>(a4.x, a4.y);
    }
};

// FP32, 12 reals: 3 float4 planes, row 2 reconstructed
struct L32_12 {
    typedef float real;
    typedef F32S store;
    static constexpr const char *name = "f32_12";
    static constexpr int planes = 3;
    static constexpr int reals = 12;
    static constexpr int bytes = 48;
    const float4 *__restrict__ p;
    int Vh;
    __device__ __forceinline__ void load(int mu, int par, int k, su3m<float> &u, int eta) const
    {
        const float4 *b = p + (size_t)((mu * 2 + par) * 3) * Vh + k;
        float4 a0 = __ldg(b), a1 = __ldg(b + Vh), a2 = __ldg(b + 2 * (size_t)Vh);
        u.e[0][0] = mk<float>(a0.x, a0.y); u.e[0][1] = mk<float>(a0.z, a0.w);
        u.e[0][2] = mk<float>(a1.x, a1.y); u.e[1][0] = mk<float>(a1.z, a1.w);
        u.e[1][1] = mk<float>(a2.x, a2.y); u.e[1][2] = mk<float>(a2.z, a2.w);
        reconstruct_row2<float>(u, (float)eta);
    }
};

// Half precision, 12 reals, two loads per link: a 16-byte plane (u00 u01 u02 u10 as __half2)
// and an 8-byte plane (u11 u12) that follows all 16-byte ones; row 2 rebuilt in FP32.  SU(3)
// entries (times the +-1 phases) lie in [-1, 1], so no scale is stored; the spinors that go
// with these links are half with a per-site scale (H16S).
struct L16_12 {
    typedef float real;
    typedef H16S store;
    static constexpr const char *name = "f16_12";
    static constexpr int planes = 2;
    static constexpr int reals = 12;
    static constexpr int bytes = 24;
    const uint4 *__restrict__ p;
    int Vh;
    __device__ __forceinline__ static cpx<float> h2c(unsigned w)
    {
        const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&w));
        return mk<float>(f.x, f.y);
    }
    __device__ __forceinline__ void load(int mu, int par, int k, su3m<float> &u, int eta) const
    {
        const size_t i = (size_t)(mu * 2 + par) * Vh + k;
        const uint4 a = __ldg(p + i);
        const uint2 b = __ldg(reinterpret_cast<const uint2 *>(p + (size_t)8 * Vh) + i);
        u.e[0][0] = h2c(a.x); u.e[0][1] = h2c(a.y);
        u.e[0][2] = h2c(a.z); u.e[1][0] = h2c(a.w);
        u.e[1][1] = h2c(b.x); u.e[1][2] = h2c(b.y);
        reconstruct_row2<float>(u, (float)eta);
    }
};

// ------------------------------------------------------------------ spinor formats
template <typename R> struct SpinorT;
template <> struct SpinorT<double> { typedef double2 elem; };
template <> struct SpinorT<float> { typedef float2 elem; };

template <typename R>
__device__ __forceinline__ vec3<R> load_spinor(const typename SpinorT<R>::elem *__restrict__ v, int Vh, int k)
{
    vec3<R> r;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        typename SpinorT<R>::elem a = __ldg(v + (size_t)c * Vh + k);
        r.c[c] = mk<R>(a.x, a.y);
    }
    return r;
}

template <typename R>
__device__ __forceinline__ void store_spinor(typename SpinorT<R>::elem *v, int Vh, int k, const vec3<R> &r)
{
#pragma unroll
    for (int c = 0; c < 3; c++) {
        typename SpinorT<R>::elem a;
        a.x = r.c[c].re;
        a.y = r.c[c].im;
        v[(size_t)c * Vh + k] = a;
    }
}

// Storage policies: elem is the array element type, planes the elements per site of one
// spinor (a spinor of parity p occupies planes * Vh elements; consecutive RHS are `stride`
// elements apart with stride >= planes * Vh).
struct F64S {
    typedef double real;
    typedef double2 elem;
    static constexpr int planes = 3;
    static constexpr bool soa = true;  // plane c of site k at c * Vh + k
    static constexpr int pack = 1;    // right-hand sides per element (PackS)
    template <typename R>
    __device__ __forceinline__ static vec3<R> load(const elem *__restrict__ v, int Vh, int k)
    {
        const vec3<double> d = load_spinor<double>(v, Vh, k);
        vec3<R> r;
#pragma unroll
        for (int c = 0; c < 3; c++) r.c[c] = mk<R>((R)d.c[c].re, (R)d.c[c].im);
        return r;
    }
    template <typename R>
    __device__ __forceinline__ static void store(elem *v, int Vh, int k, const vec3<R> &r)
    {
        vec3<double> d;
#pragma unroll
        for (int c = 0; c < 3; c++) d.c[c] = mk<double>((double)r.c[c].re, (double)r.c[c].im);
        store_spinor<double>(v, Vh, k, d);
    }
    // the same from memory that __ldg cannot address (shared), planes pstride elements apart
    template <typename R>
    __device__ __forceinline__ static vec3<R> load_plain(const elem *v, int pstride, int k)
    {
        vec3<R> r;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const elem a = v[c * pstride + k];
            r.c[c] = mk<R>((R)a.x, (R)a.y);
        }
        return r;
    }
};

struct F32S {
    typedef float real;
    typedef float2 elem;
    static constexpr int planes = 3;
    static constexpr bool soa = true;
    static constexpr int pack = 1;
    template <typename R>
    __device__ __forceinline__ static vec3<R> load(const elem *__restrict__ v, int Vh, int k)
    {
        const vec3<float> f = load_spinor<float>(v, Vh, k);
        vec3<R> r;
#pragma unroll
        for (int c = 0; c < 3; c++) r.c[c] = mk<R>((R)f.c[c].re, (R)f.c[c].im);
        return r;
    }
    template <typename R>
    __device__ __forceinline__ static void store(elem *v, int Vh, int k, const vec3<R> &r)
    {
        vec3<float> f;
#pragma unroll
        for (int c = 0; c < 3; c++) f.c[c] = mk<float>((float)r.c[c].re, (float)r.c[c].im);
        store_spinor<float>(v, Vh, k, f);
    }
    template <typename R>
    __device__ __forceinline__ static vec3<R> load_plain(const elem *v, int pstride, int k)
    {
        vec3<R> r;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const elem a = v[c * pstride + k];
            r.c[c] = mk<R>((R)a.x, (R)a.y);
        }
        return r;
    }
};

// The reference's host layout (Vec3 arrays, lib/Tools/vec3.h): the 3 complex numbers of a site
// consecutive, sites in half-index order.  A warp's 32 sites are 1536 contiguous bytes, so its
// loads stay coalesced; the host-buffer Dslash reads and writes it without conversion kernels.
struct A64S {
    typedef double real;
    typedef double2 elem;
    static constexpr int planes = 3;
    static constexpr bool soa = false;
    static constexpr int pack = 1;
    template <typename R>
    __device__ __forceinline__ static vec3<R> load(const elem *__restrict__ v, int, int k)
    {
        vec3<R> r;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const elem a = __ldg(v + (size_t)3 * k + c);
            r.c[c] = mk<R>((R)a.x, (R)a.y);
        }
        return r;
    }
    template <typename R>
    __device__ __forceinline__ static void store(elem *v, int, int k, const vec3<R> &r)
    {
#pragma unroll
        for (int c = 0; c < 3; c++) v[(size_t)3 * k + c] = make_double2((double)r.c[c].re, (double)r.c[c].im);
    }
    template <typename R>
    __device__ __forceinline__ static vec3<R> load_plain(const elem *v, int, int k)
    {
        vec3<R> r;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const elem a = v[3 * k + c];
            r.c[c] = mk<R>((R)a.x, (R)a.y);
        }
        return r;
    }
};

// Half precision with a per-site scale, one 16-byte vector per site: words x, y, z hold the
// three colour components as __half2 divided by the site's largest |real or imaginary part|,
// word w holds that scale as a float (16 bytes per site instead of 24 in FP32, and one load
// instruction per neighbour spinor).
struct H16S {
    typedef float real;
    typedef uint4 elem;
    static constexpr int planes = 1;
    static constexpr bool soa = true;
    static constexpr int pack = 1;
    __device__ __forceinline__ static float2 h2f(unsigned w) { return __half22float2(*reinterpret_cast<const __half2 *>(&w)); }
    __device__ __forceinline__ static unsigned f2h(float a, float b)
    {
        const __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<const unsigned *>(&h);
    }
    template <typename R>
    __device__ __forceinline__ static vec3<R> load(const elem *__restrict__ v, int, int k)
    {
        return decode<R>(__ldg(v + k));
    }
    template <typename R>
    __device__ __forceinline__ static vec3<R> load_plain(const elem *v, int, int k)
    {
        return decode<R>(v[k]);
    }
    template <typename R>
    __device__ __forceinline__ static vec3<R> decode(const uint4 q)
    {
        const float nrm = __uint_as_float(q.w);
        const float2 f0 = h2f(q.x), f1 = h2f(q.y), f2 = h2f(q.z);
        vec3<R> r;
        r.c[0] = mk<R>((R)(f0.x * nrm), (R)(f0.y * nrm));
        r.c[1] = mk<R>((R)(f1.x * nrm), (R)(f1.y * nrm));
        r.c[2] = mk<R>((R)(f2.x * nrm), (R)(f2.y * nrm));
        return r;
    }
    template <typename R>
    __device__ __forceinline__ static void store(elem *v, int, int k, const vec3<R> &r)
    {
        float m = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) m = fmaxf(m, fmaxf(fabsf((float)r.c[c].re), fabsf((float)r.c[c].im)));
        // a site whose largest component is below the smallest normal float is stored as zero:
        // 1/m would overflow to inf there and turn the halves into inf or NaN
        if (!(m >= FLT_MIN)) m = 0.f;
        const float inv = m > 0.f ? 1.f / m : 0.f;
        uint4 q;
        q.x = f2h((float)r.c[0].re * inv, (float)r.c[0].im * inv);
        q.y = f2h((float)r.c[1].re * inv, (float)r.c[1].im * inv);
        q.z = f2h((float)r.c[2].re * inv, (float)r.c[2].im * inv);
        q.w = __float_as_uint(m);
        v[k] = q;
    }
};

// asynchronous global -> shared copy of one element (cp.async: no registers held while in flight)
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void *smem, const void *gmem)
{
    static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async copies 4, 8 or 16 bytes");
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    const size_t ga = __cvta_generic_to_global(gmem);
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(ga) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(ga), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ------------------------------------------------------------------ packed right-hand sides
// A batch of right-hand sides stored P at a time: element (pack q, colour c, site k) holds the P
// complex numbers of RHS qP .. qP+P-1 contiguously at element index (q*3 + c)*Vh + k, consecutive
// packs `stride` elements apart (stride >= 3 Vh).  One 16- or 32-byte load then brings P
// right-hand sides of a colour and site, where one-plane-per-RHS storage needs P 8- or 16-byte
// loads: fewer load instructions, more bytes in flight per instruction.  (P = 1 is the plane
// layout of F64S / F32S.)
template <typename R, int P> struct __align__(P * 2 * sizeof(R)) PackElem { R v[2 * P]; };

template <typename R, int P> struct PackIO;
// ld: read-only path (data the kernel does not write); ldc: coherent load (read-modify-write)
template <typename R> struct PackIO<R, 1> {
    __device__ __forceinline__ static void ld(const PackElem<R, 1> *e, cpx<R> (&o)[1])
    {
        const typename SpinorT<R>::elem a = __ldg(reinterpret_cast<const typename SpinorT<R>::elem *>(e));
        o[0] = mk<R>(a.x, a.y);
    }
    __device__ __forceinline__ static void ldc(const PackElem<R, 1> *e, cpx<R> (&o)[1])
    {
        const typename SpinorT<R>::elem a = *reinterpret_cast<const typename SpinorT<R>::elem *>(e);
        o[0] = mk<R>(a.x, a.y);
    }
    __device__ __forceinline__ static void st(PackElem<R, 1> *e, const cpx<R> (&o)[1])
    {
        typename SpinorT<R>::elem a;
        a.x = o[0].re;
        a.y = o[0].im;
        *reinterpret_cast<typename SpinorT<R>::elem *>(e) = a;
    }
};
template <> struct PackIO<float, 2> {
    __device__ __forceinline__ static void ld(const PackElem<float, 2> *e, cpx<float> (&o)[2])
    {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(e));
        o[0] = mk<float>(a.x, a.y);
        o[1] = mk<float>(a.z, a.w);
    }
    __device__ __forceinline__ static void ldc(const PackElem<float, 2> *e, cpx<float> (&o)[2])
    {
        const float4 a = *reinterpret_cast<const float4 *>(e);
        o[0] = mk<float>(a.x, a.y);
        o[1] = mk<float>(a.z, a.w);
    }
    __device__ __forceinline__ static void st(PackElem<float, 2> *e, const cpx<float> (&o)[2])
    {
        *reinterpret_cast<float4 *>(e) = make_float4(o[0].re, o[0].im, o[1].re, o[1].im);
    }
};
template <> struct PackIO<float, 4> {  // 32-byte accesses (sm_100)
    __device__ __forceinline__ static void ld(const PackElem<float, 4> *e, cpx<float> (&o)[4])
    {
        float a[8];
        asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(a[4]), "=f"(a[5]), "=f"(a[6]), "=f"(a[7])
                     : "l"(e));
#pragma unroll
        for (int i = 0; i < 4; i++) o[i] = mk<float>(a[2 * i], a[2 * i + 1]);
    }
    __device__ __forceinline__ static void ldc(const PackElem<float, 4> *e, cpx<float> (&o)[4])
    {
        float a[8];
        asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(a[4]), "=f"(a[5]), "=f"(a[6]), "=f"(a[7])
                     : "l"(e)
                     : "memory");
#pragma unroll
        for (int i = 0; i < 4; i++) o[i] = mk<float>(a[2 * i], a[2 * i + 1]);
    }
    __device__ __forceinline__ static void st(PackElem<float, 4> *e, const cpx<float> (&o)[4])
    {
        asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(e), "f"(o[0].re), "f"(o[0].im), "f"(o[1].re),
                     "f"(o[1].im), "f"(o[2].re), "f"(o[2].im), "f"(o[3].re), "f"(o[3].im)
                     : "memory");
    }
};
template <> struct PackIO<double, 2> {  // 32-byte accesses (sm_100)
    __device__ __forceinline__ static void ld(const PackElem<double, 2> *e, cpx<double> (&o)[2])
    {
        double a[4];
        asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a[0]), "=d"(a[1]), "=d"(a[2]), "=d"(a[3]) : "l"(e));
        o[0] = mk<double>(a[0], a[1]);
        o[1] = mk<double>(a[2], a[3]);
    }
    __device__ __forceinline__ static void ldc(const PackElem<double, 2> *e, cpx<double> (&o)[2])
    {
        double a[4];
        asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a[0]), "=d"(a[1]), "=d"(a[2]), "=d"(a[3]) : "l"(e) : "memory");
        o[0] = mk<double>(a[0], a[1]);
        o[1] = mk<double>(a[2], a[3]);
    }
    __device__ __forceinline__ static void st(PackElem<double, 2> *e, const cpx<double> (&o)[2])
    {
        asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(e), "d"(o[0].re), "d"(o[0].im), "d"(o[1].re), "d"(o[1].im)
                     : "memory");
    }
};

// storage policy of packed spinors (the Dslash kernel reads and writes whole packs)
template <typename R, int P>
struct PackS {
    typedef R real;
    typedef PackElem<R, P> elem;
    static constexpr int planes = 3;
    static constexpr bool soa = true;
    static constexpr int pack = P;
};

// a link format whose spinors are packed P right-hand sides at a time
template <class L, int P>
struct LPack : L {
    typedef PackS<typename L::real, P> store;
};

// a*b + c*d rounded one fixed way, fma(a, b, c*d).  Left to the compiler's FMA contraction, an
// expression with two products may fuse either one, and the choice can differ between template
// instantiations: results that must be bit-identical across batch widths, launch shapes and
// storage layouts (reductions, the Dslash epilogue) use this instead.
__device__ __forceinline__ double dot2(double a, double b, double c, double d) { return __fma_rn(a, b, __dmul_rn(c, d)); }
__device__ __forceinline__ float dot2(float a, float b, float c, float d) { return __fmaf_rn(a, b, __fmul_rn(c, d)); }

// ------------------------------------------------------------------ SU(3) x vector
// acc += U v
template <typename R>
__device__ __forceinline__ void mv_acc(const su3m<R> &u, const vec3<R> &v, vec3<R> &acc)
{
#pragma unroll
    for (int i = 0; i < 3; i++) {
        cpx<R> s = acc.c[i];
        s = cmadd(u.e[i][0], v.c[0], s);
        s = cmadd(u.e[i][1], v.c[1], s);
        s = cmadd(u.e[i][2], v.c[2], s);
        acc.c[i] = s;
    }
}

// acc -= U^dag v
template <typename R>
__device__ __forceinline__ void mdv_sub(const su3m<R> &u, const vec3<R> &v, vec3<R> &acc)
{
#pragma unroll
    for (int i = 0; i < 3; i++) {
        cpx<R> s = mk<R>(0, 0);
        s = cjmadd(u.e[0][i], v.c[0], s);
        s = cjmadd(u.e[1][i], v.c[1], s);
        s = cjmadd(u.e[2][i], v.c[2], s);
        acc.c[i] = acc.c[i] - s;
    }
}

// ------------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of N values per thread; result valid in thread 0.  smem: N*32 doubles.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double *smem)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < N; j++) v[j] = warp_sum(v[j]);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < N; j++) smem[j * 32 + wid] = v[j];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int j = 0; j < N; j++) {
            double a = (lane < nw) ? smem[j * 32 + lane] : 0.0;
            v[j] = warp_sum(a);
        }
    }
    __syncthreads();
}

// Grid-wide deterministic reduction whose result does not depend on the launch's block size.
// Sites are summed in fixed chunks of RED_CHUNK = 128 consecutive threads: every thread parks
// its N values in shared memory; value j of a chunk is reduced by one warp, lane l adding
// threads l, l+32, l+64, l+96 in that order before a shuffle tree (one shuffle tree per value
// and chunk instead of one per value and warp).  Every tile of blockDim threads (blockDim 128 or
// 256) writes one partial per chunk it covers (reduce_tile); after its last tile each block takes
// a ticket, and the last block to finish sums the chunk partials with its first 128 threads
// (thread t takes chunks t, t+128, ... in order), then a shuffle tree per warp and the 4 warp
// sums in order, re-arms the ticket and hands the totals to fin(), which every thread of that
// block calls (a finaliser may split its work across them) (reduce_last).  Neither the block
// size nor the number of tiles a block walks changes a sum, so a batched launch (NR right-hand
// sides, 128-thread blocks) reduces each RHS bit for bit as a single-RHS launch (256-thread
// blocks) does, and a persistent grid as one block per tile does.  All threads of every block
// must call both parts.  partials: red_chunks(n) * N doubles.
struct NoFin {
    __device__ void operator()(const double *) const {}
};

constexpr int RED_CHUNK = 128;
constexpr int RED_BLOCK_MAX = 256;

// number of chunk partials a reduction over n threads may write, for blocks of 128 or 256
__host__ __device__ __forceinline__ long red_chunks(long n) { return 2 * ((n + 255) / 256); }

// Part 1, once per tile of blockDim.x threads (tile = blockIdx.x for one tile per block; a
// persistent block calls it for each of its tiles): the chunk partials of the tile.  Ends with a
// barrier, so the caller may reuse shared memory afterwards.
template <int N>
__device__ __forceinline__ void reduce_tile(double (&v)[N], double *partials, int tile)
{
    __shared__ double sm[N][RED_BLOCK_MAX];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int cpb = blockDim.x / RED_CHUNK;
#pragma unroll
    for (int j = 0; j < N; j++) sm[j][threadIdx.x] = v[j];
    __syncthreads();
    {
        const int c = wid >> 2, wl = wid & 3, base = c * RED_CHUNK;
        for (int j = wl; j < N; j += 4) {
            double t = sm[j][base + lane];
            t += sm[j][base + lane + 32];
            t += sm[j][base + lane + 64];
            t += sm[j][base + lane + 96];
            t = warp_sum(t);
            if (lane == 0) partials[((size_t)tile * cpb + c) * N + j] = t;
        }
    }
    __syncthreads();
}

// Part 2, once per block after its last tile: the last block to arrive (atomic ticket) sums the
// nch chunk partials and calls fin().  The block's partials were ordered before this by the
// barrier that ends reduce_tile; thread 0's fence makes them visible before its ticket.
template <int N, class FIN>
__device__ __forceinline__ void reduce_last(double *partials, unsigned *ticket, int nch, const FIN &fin)
{
    __shared__ int am_last;
    __shared__ double wsum[N][4];
    __shared__ double tot[N];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double acc[N];
#pragma unroll
    for (int j = 0; j < N; j++) acc[j] = 0.0;
    if (threadIdx.x < RED_CHUNK) {
        // chunks t, t+128, ... added in that order; the loads of B chunks are issued together
        constexpr int B = (N <= 4) ? 8 : 4;
        int i = threadIdx.x;
        for (; i + (B - 1) * RED_CHUNK < nch; i += B * RED_CHUNK) {
            double q[B][N];
#pragma unroll
            for (int u = 0; u < B; u++)
#pragma unroll
                for (int j = 0; j < N; j++) q[u][j] = __ldcg(partials + (size_t)(i + u * RED_CHUNK) * N + j);
#pragma unroll
            for (int u = 0; u < B; u++)
#pragma unroll
                for (int j = 0; j < N; j++) acc[j] += q[u][j];
        }
        for (; i < nch; i += RED_CHUNK)
#pragma unroll
            for (int j = 0; j < N; j++) acc[j] += __ldcg(partials + (size_t)i * N + j);
    }
#pragma unroll
    for (int j = 0; j < N; j++) acc[j] = warp_sum(acc[j]);
    if (lane == 0 && wid < 4)
#pragma unroll
        for (int j = 0; j < N; j++) wsum[j][wid] = acc[j];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < N; j++) {
            double t = wsum[j][0];
            t += wsum[j][1];
            t += wsum[j][2];
            t += wsum[j][3];
            tot[j] = t;
        }
        *ticket = 0;
    }
    __syncthreads();
    fin(tot);
}

template <int N, class FIN>
__device__ __forceinline__ void reduce_finalize(double (&v)[N], double *partials, unsigned *ticket, const FIN &fin)
{
    reduce_tile<N>(v, partials, blockIdx.x);
    reduce_last<N>(partials, ticket, (int)gridDim.x * (int)(blockDim.x / RED_CHUNK), fin);
}

}  // namespace rhmc
