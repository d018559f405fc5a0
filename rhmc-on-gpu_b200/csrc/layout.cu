// layout.cu -- conversions between the reference CPU layouts and the device layouts, the
// derived link formats, and the device-side geometry tables.
#include "context.h"
#include "kernels.h"

namespace rhmc {

// ------------------------------------------------------------------ geometry tables
// table[num + mu*V] = nnm[num][mu], table[num + (4+mu)*V] = nnp[num][mu]
// (make_shift_table, lib/Tools/Packer/packer.cc:415-439), eta[num + mu*V]
// (init_geo, lib/Main/Geometry/geometry.cc:107-153); both bit-exact.
__global__ void geometry_kernel(Geom g, int *table, int *eta)
{
    const long V = 2L * g.Vh;
    const long num = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (num >= V) return;
    const int p = num >= g.Vh;
    const int k = (int)(num - (long)p * g.Vh);
    const Site s = site_of(g, p, k);
    const long o = (long)(1 - p) * g.Vh;
    for (int mu = 0; mu < 4; mu++) {
        if (table) {
            table[num + mu * V] = (int)(o + neighbour(g, s, mu, -1));
            table[num + (4 + mu) * V] = (int)(o + neighbour(g, s, mu, +1));
        }
        if (eta) eta[num + mu * V] = eta_of(g, s, mu);
    }
}

// ------------------------------------------------------------------ gauge field
// reference AoS complex[4V][3][3] (index mu*V + p*Vh + k) <-> master [mu][p][9][Vh] double2
__global__ void gauge_from_ref_kernel(Geom g, double2 *U, const double2 *ref)
{
    const long Vh = g.Vh;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // over 4V links
    if (i >= 8 * Vh) return;
    const long mu = i / (2 * Vh), rem = i % (2 * Vh), p = rem / Vh, k = rem % Vh;
    const double2 *src = ref + i * 9;
    double2 *dst = U + ((mu * 2 + p) * 9) * Vh + k;
#pragma unroll
    for (int e = 0; e < 9; e++) dst[e * Vh] = src[e];
}

__global__ void gauge_to_ref_kernel(Geom g, double2 *ref, const double2 *U)
{
    const long Vh = g.Vh;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 8 * Vh) return;
    const long mu = i / (2 * Vh), rem = i % (2 * Vh), p = rem / Vh, k = rem % Vh;
    const double2 *src = U + ((mu * 2 + p) * 9) * Vh + k;
#pragma unroll
    for (int e = 0; e < 9; e++) ref[i * 9 + e] = src[e * Vh];
}

// master -> derived link formats
__global__ void derive_links_kernel(Geom g, const double2 *U, double2 *U64_12, float4 *U32_18, float4 *U32_12, uint4 *U16_12)
{
    const long Vh = g.Vh;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 8 * Vh) return;
    const long mp = i / Vh, k = i % Vh;  // mp = mu*2 + p
    const double2 *src = U + mp * 9 * Vh + k;
    double2 e[9];
#pragma unroll
    for (int j = 0; j < 9; j++) e[j] = src[j * Vh];
    if (U64_12) {
#pragma unroll
        for (int j = 0; j < 6; j++) U64_12[(mp * 6 + j) * Vh + k] = e[j];
    }
    if (U32_18) {
#pragma unroll
        for (int j = 0; j < 4; j++)
            U32_18[(mp * 4 + j) * Vh + k] = make_float4((float)e[2 * j].x, (float)e[2 * j].y, (float)e[2 * j + 1].x, (float)e[2 * j + 1].y);
        float2 *tail = reinterpret_cast<float2 *>(U32_18 + 32 * Vh);
        tail[mp * Vh + k] = make_float2((float)e[8].x, (float)e[8].y);
    }
    if (U32_12) {
#pragma unroll
        for (int j = 0; j < 3; j++)
            U32_12[(mp * 3 + j) * Vh + k] = make_float4((float)e[2 * j].x, (float)e[2 * j].y, (float)e[2 * j + 1].x, (float)e[2 * j + 1].y);
    }
    if (U16_12) {
        unsigned w[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
            const __half2 h = __floats2half2_rn((float)e[j].x, (float)e[j].y);
            w[j] = *reinterpret_cast<const unsigned *>(&h);
        }
        U16_12[mp * Vh + k] = make_uint4(w[0], w[1], w[2], w[3]);
        reinterpret_cast<uint2 *>(U16_12 + 8 * Vh)[mp * Vh + k] = make_uint2(w[4], w[5]);
    }
}

// ------------------------------------------------------------------ algebra fields
// full 3x3 (reference) <-> 8 reals [mu][p][8][Vh].  Hermitian (momenta): p01, p02, p12,
// re p00, re p11; anti-hermitian (ipdot): a01, a02, a12, im a00, im a11 -- the same
// elements the reference packs (lib/Tools/Packer/packer.cc:443-566).
__global__ void algebra_from_ref_kernel(Geom g, double *A, const double2 *ref, int antiherm)
{
    const long Vh = g.Vh;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 8 * Vh) return;
    const long mp = i / Vh, k = i % Vh;
    const double2 *m = ref + i * 9;
    double *d = A + mp * 8 * Vh + k;
    d[0] = m[1].x; d[Vh] = m[1].y;
    d[2 * Vh] = m[2].x; d[3 * Vh] = m[2].y;
    d[4 * Vh] = m[5].x; d[5 * Vh] = m[5].y;
    d[6 * Vh] = antiherm ? m[0].y : m[0].x;
    d[7 * Vh] = antiherm ? m[4].y : m[4].x;
}

__global__ void algebra_to_ref_kernel(Geom g, double2 *ref, const double *A, int antiherm)
{
    const long Vh = g.Vh;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 8 * Vh) return;
    const long mp = i / Vh, k = i % Vh;
    const double *d = A + mp * 8 * Vh + k;
    double2 *m = ref + i * 9;
    const double2 a01 = make_double2(d[0], d[Vh]), a02 = make_double2(d[2 * Vh], d[3 * Vh]), a12 = make_double2(d[4 * Vh], d[5 * Vh]);
    const double d0 = d[6 * Vh], d1 = d[7 * Vh], d2 = -d0 - d1;
    if (antiherm) {
        m[0] = make_double2(0.0, d0); m[4] = make_double2(0.0, d1); m[8] = make_double2(0.0, d2);
        m[1] = a01; m[2] = a02; m[5] = a12;
        m[3] = make_double2(-a01.x, a01.y); m[6] = make_double2(-a02.x, a02.y); m[7] = make_double2(-a12.x, a12.y);
    } else {
        m[0] = make_double2(d0, 0.0); m[4] = make_double2(d1, 0.0); m[8] = make_double2(d2, 0.0);
        m[1] = a01; m[2] = a02; m[5] = a12;
        m[3] = make_double2(a01.x, -a01.y); m[6] = make_double2(a02.x, -a02.y); m[7] = make_double2(a12.x, -a12.y);
    }
}

// ------------------------------------------------------------------ spinors
template <typename E>
__global__ void spinor_to_internal_kernel(long Vh, int n, E *dst, const double2 *src)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // over n*Vh
    if (i >= n * Vh) return;
    const long r = i / Vh, k = i % Vh;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double2 v = src[i * 3 + c];
        E o;
        o.x = v.x;
        o.y = v.y;
        dst[(r * 3 + c) * Vh + k] = o;
    }
}

template <typename E>
__global__ void spinor_from_internal_kernel(long Vh, int n, double2 *dst, const E *src)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * Vh) return;
    const long r = i / Vh, k = i % Vh;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        E v = src[(r * 3 + c) * Vh + k];
        dst[i * 3 + c] = make_double2(v.x, v.y);
    }
}

// reference layout <-> half precision with per-site scale (H16S, Vh 16-byte vectors per spinor)
__global__ void spinor_to_half_kernel(long Vh, int n, uint4 *dst, const double2 *src)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * Vh) return;
    const long r = i / Vh, k = i % Vh;
    vec3<double> v;
#pragma unroll
    for (int c = 0; c < 3; c++) v.c[c] = mk<double>(src[i * 3 + c].x, src[i * 3 + c].y);
    H16S::store<double>(dst + r * Vh, (int)Vh, (int)k, v);
}

__global__ void spinor_from_half_kernel(long Vh, int n, double2 *dst, const uint4 *src)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * Vh) return;
    const long r = i / Vh, k = i % Vh;
    const vec3<double> v = H16S::load<double>(src + r * Vh, (int)Vh, (int)k);
#pragma unroll
    for (int c = 0; c < 3; c++) dst[i * 3 + c] = make_double2(v.c[c].re, v.c[c].im);
}

// ------------------------------------------------------------------ host launchers
int grid_for(long n, int block) { return (int)((n + block - 1) / block); }

void launch_geometry(rhmc_ctx *c, int *table, int *eta)
{
    geometry_kernel<<<grid_for(2L * c->Vh, 256), 256, 0, c->stream>>>(c->g, table, eta);
    c->launches++;
}

void launch_gauge_from_ref(rhmc_ctx *c, const double *ref)
{
    gauge_from_ref_kernel<<<grid_for(8L * c->Vh, 256), 256, 0, c->stream>>>(c->g, c->U64, reinterpret_cast<const double2 *>(ref));
    c->launches++;
}

void launch_gauge_to_ref(rhmc_ctx *c, double *ref)
{
    gauge_to_ref_kernel<<<grid_for(8L * c->Vh, 256), 256, 0, c->stream>>>(c->g, reinterpret_cast<double2 *>(ref), c->U64);
    c->launches++;
}

void launch_algebra_from_ref(rhmc_ctx *c, double *A, const double *ref, int antiherm)
{
    algebra_from_ref_kernel<<<grid_for(8L * c->Vh, 256), 256, 0, c->stream>>>(c->g, A, reinterpret_cast<const double2 *>(ref), antiherm);
    c->launches++;
}

void launch_algebra_to_ref(rhmc_ctx *c, double *ref, const double *A, int antiherm)
{
    algebra_to_ref_kernel<<<grid_for(8L * c->Vh, 256), 256, 0, c->stream>>>(c->g, reinterpret_cast<double2 *>(ref), A, antiherm);
    c->launches++;
}

void launch_spinor_to_internal(rhmc_ctx *c, int fmt, void *dst, const double *src, int n)
{
    const int grid = grid_for((long)n * c->Vh, 256);
    if (fmt == RHMC_LINKS_F16_12) spinor_to_half_kernel<<<grid, 256, 0, c->stream>>>(c->Vh, n, (uint4 *)dst, (const double2 *)src);
    else if (fmt_is_f64(fmt)) spinor_to_internal_kernel<double2><<<grid, 256, 0, c->stream>>>(c->Vh, n, (double2 *)dst, (const double2 *)src);
    else spinor_to_internal_kernel<float2><<<grid, 256, 0, c->stream>>>(c->Vh, n, (float2 *)dst, (const double2 *)src);
    c->launches++;
}

void launch_spinor_from_internal(rhmc_ctx *c, int fmt, double *dst, const void *src, int n)
{
    const int grid = grid_for((long)n * c->Vh, 256);
    if (fmt == RHMC_LINKS_F16_12) spinor_from_half_kernel<<<grid, 256, 0, c->stream>>>(c->Vh, n, (double2 *)dst, (const uint4 *)src);
    else if (fmt_is_f64(fmt)) spinor_from_internal_kernel<double2><<<grid, 256, 0, c->stream>>>(c->Vh, n, (double2 *)dst, (const double2 *)src);
    else spinor_from_internal_kernel<float2><<<grid, 256, 0, c->stream>>>(c->Vh, n, (double2 *)dst, (const float2 *)src);
    c->launches++;
}

static cudaError_t ensure_derived(rhmc_ctx *c, int fmt)
{
    if (c->derived_valid[fmt]) return cudaSuccess;
    void *p = nullptr;
    cudaError_t e = cudaSuccess;
    const size_t Vh = c->Vh;
    if (fmt == RHMC_LINKS_F64_12 && !c->U64_12) e = cudaMalloc(&p, 8 * 6 * Vh * sizeof(double2)), c->U64_12 = (double2 *)p;
    if (fmt == RHMC_LINKS_F32_18 && !c->U32_18) e = cudaMalloc(&p, 8 * 4 * Vh * sizeof(float4) + 8 * Vh * sizeof(float2)), c->U32_18 = (float4 *)p;
    if (fmt == RHMC_LINKS_F32_12 && !c->U32_12) e = cudaMalloc(&p, 8 * 3 * Vh * sizeof(float4)), c->U32_12 = (float4 *)p;
    if (fmt == RHMC_LINKS_F16_12 && !c->U16_12) e = cudaMalloc(&p, 8 * Vh * (sizeof(uint4) + sizeof(uint2))), c->U16_12 = (uint4 *)p;
    if (e != cudaSuccess) return e;
    derive_links_kernel<<<grid_for(8L * c->Vh, 256), 256, 0, c->stream>>>(
        c->g, c->U64, fmt == RHMC_LINKS_F64_12 ? c->U64_12 : nullptr, fmt == RHMC_LINKS_F32_18 ? c->U32_18 : nullptr,
        fmt == RHMC_LINKS_F32_12 ? c->U32_12 : nullptr, fmt == RHMC_LINKS_F16_12 ? c->U16_12 : nullptr);
    c->launches++;
    c->derived_valid[fmt] = true;
    return cudaGetLastError();
}

void invalidate_links(rhmc_ctx *c)
{
    c->derived_valid[RHMC_LINKS_F64_12] = c->derived_valid[RHMC_LINKS_F32_18] = c->derived_valid[RHMC_LINKS_F32_12] = false;
    c->derived_valid[RHMC_LINKS_F16_12] = false;
}

cudaError_t links_f64_18(rhmc_ctx *c, L64_18 *lf) { lf->p = c->U64; lf->Vh = (int)c->Vh; return cudaSuccess; }
cudaError_t links_f64_12(rhmc_ctx *c, L64_12 *lf) { cudaError_t e = ensure_derived(c, RHMC_LINKS_F64_12); lf->p = c->U64_12; lf->Vh = (int)c->Vh; return e; }
cudaError_t links_f32_18(rhmc_ctx *c, L32_18 *lf) { cudaError_t e = ensure_derived(c, RHMC_LINKS_F32_18); lf->p = c->U32_18; lf->Vh = (int)c->Vh; return e; }
cudaError_t links_f32_12(rhmc_ctx *c, L32_12 *lf) { cudaError_t e = ensure_derived(c, RHMC_LINKS_F32_12); lf->p = c->U32_12; lf->Vh = (int)c->Vh; return e; }
cudaError_t links_f16_12(rhmc_ctx *c, L16_12 *lf) { cudaError_t e = ensure_derived(c, RHMC_LINKS_F16_12); lf->p = c->U16_12; lf->Vh = (int)c->Vh; return e; }

}  // namespace rhmc
