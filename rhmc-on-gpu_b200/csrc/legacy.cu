// legacy.cu -- the reference's extern "C" GPU entry points (the lib/Cuda headers) on top of
// one library context, reading and writing the host program's packed buffers in the formats
// of lib/Tools/Packer/packer.cc.  Declared in include/rhmc_legacy.h.
//
// Device state of the reference (lib/Cuda/cuda_rhmc.cuh:73-79) and its equivalent here:
//   gauge_field_device  -> the context's FP64 link field
//   mf_device (chi)     -> g_mf: no_ps FP64 even spinors
//   smf_device (x_i)    -> g_smf: no_ps x max_approx_order FP64 even spinors, [ps][shift]
//   ipdot/momenta       -> the context's FP64 algebra fields
// Format conversions run on the GPU; the packed float buffers are staged through device
// copies.  Errors print and exit as cudaSafe does (lib/Cuda/cuda_err.cu:5-13), because these
// entry points return void like the originals; the handle API returns codes instead.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/rhmc_legacy.h"
#include "capi_util.h"
#include "context.h"
#include "kernels.h"
#include "su3.cuh"

namespace rhmc {

int gauge_force(rhmc_ctx *c, int mode);
int fermion_force(rhmc_ctx *c, int nrhs, int nshift, const double *a, const double2 *x, int mode);
int mom_update(rhmc_ctx *c, double step);
int link_update(rhmc_ctx *c, double step);
int rational_sum(rhmc_ctx *c, int nrhs, int nshift, double a0, const double *a, const double2 *x, const double2 *b, double2 *out,
                 int add);
int rdot(rhmc_ctx *c, const double2 *a, const double2 *b, long n, double *out);

static rhmc_legacy_config g_cfg;
static bool g_bound = false;
static rhmc_ctx *g_ctx = nullptr;
static double2 *g_mf = nullptr, *g_smf = nullptr;

[[noreturn]] static void die(const char *where)
{
    fprintf(stderr, "librhmc_b200 legacy %s: %s\n", where, rhmc_last_error());
    exit(-1);
}

#define LEG(call, where)                   \
    do {                                   \
        if ((call) != RHMC_OK) die(where); \
    } while (0)

// ------------------------------------------------------------------ packed formats
// gauge: float hi[12*4V] then lo[12*4V]; for link (mu, site i): three float4 at
// 4i + 12 mu V + {0, 4V, 8V}: (u00, u01), (u02, u10), (u11, u12) re/im (packer.cc:18-64)
__global__ void gauge_from_packed(Geom g, const float *__restrict__ pk, double2 *U)
{
    const long V = 2L * g.Vh, Vh = g.Vh;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const long mu = t / V, i = t % V;
    const int p = i >= Vh;
    const int k = (int)(i - p * Vh);
    const long offs = 12 * 4 * V;
    M3 u;
    double r[12];
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const long o = 4 * i + e + q * 4 * V + 12 * mu * V;
            r[q * 4 + e] = (double)pk[o] + (double)pk[offs + o];
        }
    u.e[0][0] = mk<double>(r[0], r[1]);
    u.e[0][1] = mk<double>(r[2], r[3]);
    u.e[0][2] = mk<double>(r[4], r[5]);
    u.e[1][0] = mk<double>(r[6], r[7]);
    u.e[1][1] = mk<double>(r[8], r[9]);
    u.e[1][2] = mk<double>(r[10], r[11]);
    // smartunpack_gauge reconstructs with Conf::unitarize_with_eta (packer.cc:131-134)
    const Site s = site_of(g, p, k);
    sunitarize_eta(u, (double)eta_of(g, s, (int)mu));
    store_link64(U, g.Vh, (int)mu, p, k, u);
}

__global__ void gauge_to_packed(Geom g, const double2 *__restrict__ U, float *pk)
{
    const long V = 2L * g.Vh, Vh = g.Vh;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const long mu = t / V, i = t % V;
    const int p = i >= Vh;
    const int k = (int)(i - p * Vh);
    const long offs = 12 * 4 * V;
    const M3 u = load_link64(U, g.Vh, (int)mu, p, k);
    const double r[12] = {u.e[0][0].re, u.e[0][0].im, u.e[0][1].re, u.e[0][1].im, u.e[0][2].re, u.e[0][2].im,
                          u.e[1][0].re, u.e[1][0].im, u.e[1][1].re, u.e[1][1].im, u.e[1][2].re, u.e[1][2].im};
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const long o = 4 * i + e + q * 4 * V + 12 * mu * V;
            const float hi = (float)r[q * 4 + e];
            pk[o] = hi;
            pk[offs + o] = (float)(r[q * 4 + e] - (double)hi);
        }
}

// spinor blocks: colour c of site i at base + 2i + c*V (re, im); lo part at +lo (packer.cc:278-321)
__global__ void spinor_from_packed(long Vh, const float *__restrict__ pk, long base, long lo, double2 *out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Vh) return;
    const long V = 2 * Vh;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const long o = base + 2 * i + c * V;
        out[c * Vh + i] = make_double2((double)pk[o] + (double)pk[lo + o], (double)pk[o + 1] + (double)pk[lo + o + 1]);
    }
}

__global__ void spinor_to_packed(long Vh, const double2 *__restrict__ in, long base, long lo, float *pk)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Vh) return;
    const long V = 2 * Vh;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const long o = base + 2 * i + c * V;
        const double2 v = in[c * Vh + i];
        const float hr = (float)v.x, hm = (float)v.y;
        pk[o] = hr;
        pk[o + 1] = hm;
        pk[lo + o] = (float)(v.x - (double)hr);
        pk[lo + o + 1] = (float)(v.y - (double)hm);
    }
}

// algebra: two float4 per link at 4i + 8 mu V + {0, 4V}: (re01, im01, re02, im02),
// (re12, im12, d0, d1) -- the same 8 reals as the device planes (packer.cc:443-566)
__global__ void alg_from_packed(long Vh, const float *__restrict__ pk, double *A)
{
    const long V = 2 * Vh;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const long mu = t / V, i = t % V;
    const int p = i >= Vh;
    const long k = i - p * Vh;
    double *d = A + ((mu * 2 + p) * 8) * Vh + k;
#pragma unroll
    for (int e = 0; e < 8; e++) d[e * Vh] = (double)pk[4 * i + (e & 3) + (e >> 2) * 4 * V + 8 * mu * V];
}

__global__ void alg_to_packed(long Vh, const double *__restrict__ A, float *pk)
{
    const long V = 2 * Vh;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const long mu = t / V, i = t % V;
    const int p = i >= Vh;
    const long k = i - p * Vh;
    const double *d = A + ((mu * 2 + p) * 8) * Vh + k;
#pragma unroll
    for (int e = 0; e < 8; e++) pk[4 * i + (e & 3) + (e >> 2) * 4 * V + 8 * mu * V] = (float)d[e * Vh];
}

__global__ void scale_kernel(long n, double2 *v, double s)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = make_double2(s * v[i].x, s * v[i].y);
}

// v = a v - w
__global__ void axmy_kernel(long n, double2 *v, double a, const double2 *__restrict__ w)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = make_double2(a * v[i].x - w[i].x, a * v[i].y - w[i].y);
}

static int stage(rhmc_ctx *c, const char *name, size_t bytes, void **p)
{
    CK(c->ws.get(name, bytes, p));
    return RHMC_OK;
}

// H2D into the staging slot; the slot is reused by the next upload only after the kernels
// queued on the same stream have consumed it (stream order)
static int upload_floats(rhmc_ctx *c, const float *h, size_t n, float **d)
{
    void *p = nullptr;
    int rc = stage(c, "leg_stage", n * sizeof(float), &p);
    if (rc) return rc;
    CK(cudaMemcpyAsync(p, h, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    *d = (float *)p;
    return RHMC_OK;
}

static int download_floats(rhmc_ctx *c, float *h, const float *d, size_t n)
{
    CK(cudaMemcpyAsync(h, d, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return RHMC_OK;
}

// ------------------------------------------------------------------ power iteration (FP64)
static int power_iteration(rhmc_ctx *c, const double2 *start, double shift_max, bool for_min, double *out)
{
    const long n = 3 * c->Vh;
    void *pv, *qv;
    CK(c->ws.get("pw_p", n * sizeof(double2), &pv));
    CK(c->ws.get("pw_q", n * sizeof(double2), &qv));
    double2 *p = (double2 *)pv, *q = (double2 *)qv;
    CK(cudaMemcpyAsync(p, start, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    double nrm2 = 0.0;
    int rc = rdot(c, p, p, n, &nrm2);
    if (rc) return rc;
    if (!(nrm2 >= 1e-9)) return fail(RHMC_ERR_ARG, "power iteration: start vector norm %g too small", sqrt(nrm2));
    double nrm = sqrt(nrm2), old, rel;
    const int grid = grid_for(n, 256);
    int it = 0;
    do {
        scale_kernel<<<grid, 256, 0, c->stream>>>(n, p, 1.0 / nrm);
        c->launches++;
        old = nrm;
        rc = rhmc_mdagm(c, RHMC_LINKS_F64_18, q, p, 0.0, 1);
        if (rc) return rc;
        if (for_min) {
            axmy_kernel<<<grid, 256, 0, c->stream>>>(n, p, shift_max, q);  // p = max p - M^dag M p
            c->launches++;
        } else {
            CK(cudaMemcpyAsync(p, q, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
        }
        if ((rc = rdot(c, p, p, n, &nrm2))) return rc;
        nrm = sqrt(nrm2);
        rel = fabs(old - nrm) / (for_min ? fabs(shift_max - nrm) : nrm);
        if (++it > 100000) return fail(RHMC_ERR_MAXITER, "power iteration did not converge");
    } while (rel > 5.0e-4);
    *out = for_min ? shift_max - nrm : nrm;
    return RHMC_OK;
}

static int find_bound(rhmc_ctx *c, const double *start_ref, double max, bool for_min, double *out)
{
    if (!c || !start_ref || !out) return fail(RHMC_ERR_ARG, "bad argument");
    void *d;
    CK(c->ws.get("pw_start", 3 * c->Vh * sizeof(double2), &d));
    int rc = rhmc_spinor_to_internal(c, RHMC_LINKS_F64_18, d, start_ref, 1, RHMC_HOST);
    if (rc) return rc;
    return power_iteration(c, (const double2 *)d, max, for_min, out);
}

static size_t spinor_elems() { return 3 * (size_t)g_ctx->Vh; }

static void need_ctx(const char *where)
{
    if (!g_bound) {
        fprintf(stderr, "librhmc_b200 legacy %s: rhmc_legacy_bind was not called\n", where);
        exit(-1);
    }
    if (!g_ctx) {
        fprintf(stderr, "librhmc_b200 legacy %s: cuda_init0 was not called\n", where);
        exit(-1);
    }
}

static void shifted_inverter(const double residual, const double *shifts, const int num_shifts, const int psferm, int *ncount,
                             int mode, int fmt, const char *where)
{
    need_ctx(where);
    if (!g_mf) {
        fprintf(stderr, "librhmc_b200 legacy %s: cuda_init1 was not called\n", where);
        exit(-1);
    }
    if (psferm < 0 || psferm >= g_cfg.no_ps || num_shifts < 1 || num_shifts > g_cfg.max_approx_order) {
        fprintf(stderr, "librhmc_b200 legacy %s: bad pseudofermion %d or shift count %d\n", where, psferm, num_shifts);
        exit(-1);
    }
    rhmc_msolve_params mp;
    memset(&mp, 0, sizeof(mp));
    mp.nshift = num_shifts;
    mp.shifts = shifts;
    mp.nrhs = 1;
    mp.residual = residual;
    mp.max_iter = g_cfg.max_cg;
    mp.mode = mode;
    mp.fmt = fmt;
    rhmc_msolve_info info;
    const size_t n = spinor_elems();
    int rc = rhmc_msolve(g_ctx, &mp, (double *)(g_smf + (size_t)psferm * g_cfg.max_approx_order * n),
                         (const double *)(g_mf + (size_t)psferm * n), &info);
    if (rc == RHMC_ERR_MAXITER) {
        *ncount = g_cfg.max_cg;  // the caller reports it and exits (cu_inverter.cc:62-69)
        return;
    }
    if (rc) die(where);
    *ncount = info.iters[0];
}

}  // namespace rhmc

using namespace rhmc;

extern "C" {

int rhmc_legacy_bind(const rhmc_legacy_config *cfg)
{
    if (!cfg) return fail(RHMC_ERR_ARG, "null config");
    if (cfg->no_ps < 1 || cfg->max_approx_order < 1 || cfg->max_approx_order > 32 || cfg->max_cg < 1)
        return fail(RHMC_ERR_ARG, "bad no_ps / max_approx_order / max_cg");
    if (!cfg->gauge_field_packed || !cfg->chi_packed || !cfg->ipdot_packed || !cfg->momenta_packed)
        return fail(RHMC_ERR_ARG, "packed buffers must be given");
    // a new binding starts from scratch: the previous context had the old constants
    if (g_ctx) {
        rhmc_destroy(g_ctx);
        g_ctx = nullptr;
        g_mf = g_smf = nullptr;
    }
    g_cfg = *cfg;
    g_bound = true;
    return RHMC_OK;
}

rhmc_ctx *rhmc_legacy_context(void) { return g_ctx; }

int rhmc_find_max(rhmc_ctx *c, const double *start, double *max) { return find_bound(c, start, 0.0, false, max); }
int rhmc_find_min(rhmc_ctx *c, const double *start, double max, double *min) { return find_bound(c, start, max, true, min); }

// cuda_init0 (lib/Cuda/cuda_init.cu:5-58): links, neighbour table and phases to the device
void cuda_init0(void)
{
    if (!g_bound) {
        fprintf(stderr, "librhmc_b200 legacy cuda_init0: rhmc_legacy_bind was not called\n");
        exit(-1);
    }
    if (!g_ctx) {
        rhmc_params p;
        p.nx = g_cfg.nx; p.ny = g_cfg.ny; p.nz = g_cfg.nz; p.nt = g_cfg.nt;
        p.ferm_temp_bc = g_cfg.ferm_temp_bc;
        p.mass = g_cfg.mass;
        p.beta = g_cfg.beta;
        p.device = g_cfg.device;
        LEG(rhmc_create(&p, &g_ctx), "cuda_init0");
        // the host geometry must be the one the kernels compute
        if (g_cfg.shift_table || g_cfg.eta) {
            std::vector<int> t(8 * g_ctx->V), e(4 * g_ctx->V);
            LEG(rhmc_geometry(g_ctx, t.data(), e.data()), "cuda_init0");
            if ((g_cfg.shift_table && memcmp(t.data(), g_cfg.shift_table, t.size() * sizeof(int))) ||
                (g_cfg.eta && memcmp(e.data(), g_cfg.eta, e.size() * sizeof(int)))) {
                fprintf(stderr, "librhmc_b200 legacy cuda_init0: host neighbour table or phases differ from the "
                                "library's even/odd geometry\n");
                exit(-1);
            }
        }
    }
    rhmc_ctx *c = g_ctx;
    float *d = nullptr;
    LEG(upload_floats(c, g_cfg.gauge_field_packed, 2 * 12 * 4 * (size_t)c->V, &d), "cuda_init0");
    gauge_from_packed<<<grid_for(4 * c->V, 256), 256, 0, c->stream>>>(c->g, d, c->U64);
    c->launches++;
    invalidate_links(c);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess) {
        fprintf(stderr, "librhmc_b200 legacy cuda_init0: CUDA error\n");
        exit(-1);
    }
}

// cuda_init1 (cuda_init.cu:61-109): chi for every pseudofermion, zeroed shifted solutions,
// ipdot and momenta
void cuda_init1(void)
{
    need_ctx("cuda_init1");
    rhmc_ctx *c = g_ctx;
    const size_t n = spinor_elems(), nps = g_cfg.no_ps;
    void *mf = nullptr, *smf = nullptr;
    LEG(stage(c, "leg_mf", nps * n * sizeof(double2), &mf), "cuda_init1");
    LEG(stage(c, "leg_smf", nps * g_cfg.max_approx_order * n * sizeof(double2), &smf), "cuda_init1");
    g_mf = (double2 *)mf;
    g_smf = (double2 *)smf;
    float *d = nullptr;
    LEG(upload_floats(c, g_cfg.chi_packed, 6 * (size_t)c->Vh * nps * 2, &d), "cuda_init1");
    for (size_t ps = 0; ps < nps; ps++)
        spinor_from_packed<<<grid_for(c->Vh, 256), 256, 0, c->stream>>>(c->Vh, d, 3 * c->V * ps, 3 * c->V * nps, g_mf + ps * n);
    cudaMemsetAsync(g_smf, 0, nps * g_cfg.max_approx_order * n * sizeof(double2), c->stream);
    LEG(upload_floats(c, g_cfg.ipdot_packed, 8 * 4 * (size_t)c->V, &d), "cuda_init1");
    alg_from_packed<<<grid_for(4 * c->V, 256), 256, 0, c->stream>>>(c->Vh, d, c->IP);
    LEG(upload_floats(c, g_cfg.momenta_packed, 8 * 4 * (size_t)c->V, &d), "cuda_init1");
    alg_from_packed<<<grid_for(4 * c->V, 256), 256, 0, c->stream>>>(c->Vh, d, c->P);
    c->launches += nps + 2;
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess) die("cuda_init1");
}

// cuda_meas_init (cuda_init.cu:112-150): one fermion into chi slot 0, zeroed solutions
void cuda_meas_init(void)
{
    need_ctx("cuda_meas_init");
    if (!g_cfg.simple_fermion_packed) die("cuda_meas_init (no simple_fermion_packed bound)");
    if (!g_mf) cuda_init1();
    rhmc_ctx *c = g_ctx;
    const size_t n = spinor_elems();
    float *d = nullptr;
    LEG(upload_floats(c, g_cfg.simple_fermion_packed, 6 * (size_t)c->Vh * 2, &d), "cuda_meas_init");
    spinor_from_packed<<<grid_for(c->Vh, 256), 256, 0, c->stream>>>(c->Vh, d, 0, 3 * c->V, g_mf);
    cudaMemsetAsync(g_smf, 0, (size_t)g_cfg.no_ps * g_cfg.max_approx_order * n * sizeof(double2), c->stream);
    c->launches++;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) die("cuda_meas_init");
}

// cuda_meas_end (cuda_init.cu:153-183): the first shifted solution back into simple_fermion_packed
void cuda_meas_end(void)
{
    need_ctx("cuda_meas_end");
    rhmc_ctx *c = g_ctx;
    void *d = nullptr;
    LEG(stage(c, "leg_stage", 6 * (size_t)c->Vh * 2 * sizeof(float), &d), "cuda_meas_end");
    spinor_to_packed<<<grid_for(c->Vh, 256), 256, 0, c->stream>>>(c->Vh, g_smf, 0, 3 * c->V, (float *)d);
    c->launches++;
    LEG(download_floats(c, g_cfg.simple_fermion_packed, (const float *)d, 6 * (size_t)c->Vh * 2), "cuda_meas_end");
}

void cuda_get_conf(void)
{
    need_ctx("cuda_get_conf");
    rhmc_ctx *c = g_ctx;
    void *d = nullptr;
    const size_t nf = 2 * 12 * 4 * (size_t)c->V;
    LEG(stage(c, "leg_stage", nf * sizeof(float), &d), "cuda_get_conf");
    gauge_to_packed<<<grid_for(4 * c->V, 256), 256, 0, c->stream>>>(c->g, c->U64, (float *)d);
    c->launches++;
    LEG(download_floats(c, g_cfg.gauge_field_packed, (const float *)d, nf), "cuda_get_conf");
}

void cuda_get_momenta(void)
{
    need_ctx("cuda_get_momenta");
    rhmc_ctx *c = g_ctx;
    void *d = nullptr;
    LEG(stage(c, "leg_stage", 8 * 4 * (size_t)c->V * sizeof(float), &d), "cuda_get_momenta");
    alg_to_packed<<<grid_for(4 * c->V, 256), 256, 0, c->stream>>>(c->Vh, c->P, (float *)d);
    c->launches++;
    LEG(download_floats(c, g_cfg.momenta_packed, (const float *)d, 8 * 4 * (size_t)c->V), "cuda_get_momenta");
}

void cuda_put_momenta(void)
{
    need_ctx("cuda_put_momenta");
    rhmc_ctx *c = g_ctx;
    float *d = nullptr;
    LEG(upload_floats(c, g_cfg.momenta_packed, 8 * 4 * (size_t)c->V, &d), "cuda_put_momenta");
    alg_from_packed<<<grid_for(4 * c->V, 256), 256, 0, c->stream>>>(c->Vh, d, c->P);
    c->launches++;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) die("cuda_put_momenta");
}

// cuda_end (cuda_init.cu:187-211): links, momenta and ipdot back to the host buffers.  The
// device fields stay allocated for the next trajectory (the reference frees and reallocates).
void cuda_end(void)
{
    need_ctx("cuda_end");
    cuda_get_conf();
    cuda_get_momenta();
    rhmc_ctx *c = g_ctx;
    void *d = nullptr;
    LEG(stage(c, "leg_stage", 8 * 4 * (size_t)c->V * sizeof(float), &d), "cuda_end");
    alg_to_packed<<<grid_for(4 * c->V, 256), 256, 0, c->stream>>>(c->Vh, c->IP, (float *)d);
    c->launches++;
    LEG(download_floats(c, g_cfg.ipdot_packed, (const float *)d, 8 * 4 * (size_t)c->V), "cuda_end");
}

void cuda_shifted_inverter(const double residual, const double *shifts, const int num_shifts, const int psferm, int *ncount)
{
    shifted_inverter(residual, shifts, num_shifts, psferm, ncount, RHMC_MSOLVE_FP32, RHMC_LINKS_F32_12, "cuda_shifted_inverter");
}

void cuda_shifted_inverter_d(const double residual, const double *shifts, const int num_shifts, const int psferm, int *ncount)
{
    shifted_inverter(residual, shifts, num_shifts, psferm, ncount, RHMC_MSOLVE_FP64, RHMC_LINKS_F64_18, "cuda_shifted_inverter_d");
}

// cuda_sol_sum (cuda_sol_sum.cu:168-221): chi = a0 chi + sum_i a_i x_i per pseudofermion, in
// place, then chi back to chi_packed
void cuda_sol_sum(const int num_shifts, const double mult_const, const double *numerators)
{
    need_ctx("cuda_sol_sum");
    rhmc_ctx *c = g_ctx;
    const size_t n = spinor_elems(), nps = g_cfg.no_ps;
    void *tmp = nullptr, *d = nullptr;
    LEG(stage(c, "leg_tmp", n * sizeof(double2), &tmp), "cuda_sol_sum");
    LEG(stage(c, "leg_stage", 6 * (size_t)c->Vh * nps * 2 * sizeof(float), &d), "cuda_sol_sum");
    for (size_t ps = 0; ps < nps; ps++) {
        LEG(rational_sum(c, 1, num_shifts, mult_const, numerators, g_smf + ps * g_cfg.max_approx_order * n, g_mf + ps * n,
                         (double2 *)tmp, 0),
            "cuda_sol_sum");
        cudaMemcpyAsync(g_mf + ps * n, tmp, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream);
        spinor_to_packed<<<grid_for(c->Vh, 256), 256, 0, c->stream>>>(c->Vh, g_mf + ps * n, 3 * c->V * ps, 3 * c->V * nps,
                                                                       (float *)d);
        c->launches++;
    }
    LEG(download_floats(c, g_cfg.chi_packed, (const float *)d, 6 * (size_t)c->Vh * nps * 2), "cuda_sol_sum");
}

// cuda_fermion_force (cuda_fermion_force.cu:346-418): ipdot = TA(U F) from the shifted
// solutions of every pseudofermion (overwrites ipdot)
void cuda_fermion_force(int num_shifts, float *numerators)
{
    need_ctx("cuda_fermion_force");
    std::vector<double> a(num_shifts);
    for (int i = 0; i < num_shifts; i++) a[i] = numerators[i];
    // shifted solutions are stored [ps][max_approx_order]; pass each pseudofermion's block
    for (int ps = 0; ps < g_cfg.no_ps; ps++)
        LEG(fermion_force(g_ctx, 1, num_shifts, a.data(), g_smf + (size_t)ps * g_cfg.max_approx_order * spinor_elems(), ps > 0),
            "cuda_fermion_force");
}

// cuda_gauge_deriv (cuda_deriv.cu:697-744): ipdot (init 0: =, init 1: +=) TA(U beta/3 staples)
void cuda_gauge_deriv(int ipdot_init)
{
    need_ctx("cuda_gauge_deriv");
    LEG(gauge_force(g_ctx, ipdot_init ? 1 : 0), "cuda_gauge_deriv");
}

void cuda_exp_su3(float step)
{
    need_ctx("cuda_exp_su3");
    LEG(link_update(g_ctx, (double)step), "cuda_exp_su3");
}

void cuda_momenta_sum_multiply(float step)
{
    need_ctx("cuda_momenta_sum_multiply");
    LEG(mom_update(g_ctx, (double)step), "cuda_momenta_sum_multiply");
}

// cuda_find_max / cuda_find_min (cuda_find_min_max.cu:69-222): start from simple_fermion_packed
// The start vector of the power iterations: findminmax packs it with the single-precision
// smartpack_fermion (findminmax.cc:161, packer.cc:156-190), which fills only the first 6*sizeh
// floats of simple_fermion_packed, and cuda_find_max/min copy only those (cuda_find_min_max.cu:
// 97-99, 172-174); whatever the rest of the buffer holds is not part of the vector.
static void start_vector(std::vector<double> &start)
{
    const long Vh = g_ctx->Vh, V = 2 * Vh;
    const float *pk = g_cfg.simple_fermion_packed;
    start.assign(6 * Vh, 0.0);
    for (long i = 0; i < Vh; i++)
        for (int c = 0; c < 3; c++) {
            start[(i * 3 + c) * 2] = (double)pk[2 * i + c * V];
            start[(i * 3 + c) * 2 + 1] = (double)pk[2 * i + c * V + 1];
        }
}

void cuda_find_max(double *max)
{
    need_ctx("cuda_find_max");
    if (!g_cfg.simple_fermion_packed) die("cuda_find_max (no simple_fermion_packed bound)");
    std::vector<double> s;
    start_vector(s);
    if (rhmc_find_max(g_ctx, s.data(), max) != RHMC_OK) {
        fprintf(stderr, "librhmc_b200 legacy cuda_find_max: %s\n", rhmc_last_error());
        exit(1);
    }
}

void cuda_find_min(double *min, const double max)
{
    need_ctx("cuda_find_min");
    if (!g_cfg.simple_fermion_packed) die("cuda_find_min (no simple_fermion_packed bound)");
    std::vector<double> s;
    start_vector(s);
    if (rhmc_find_min(g_ctx, s.data(), max, min) != RHMC_OK) die("cuda_find_min");
}

// GPUDeviceInfo (lib/Cuda/DeviceInfo/device_info.h:4-6), which the reference's main program calls
// once at start-up: selects the device and prints its properties; exits when it does not exist.
void GPUDeviceInfo(const int gpu_device)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || gpu_device < 0 || gpu_device >= n) {
        fprintf(stderr, "librhmc_b200 GPUDeviceInfo: device %d not available (%d CUDA devices)\n", gpu_device, n);
        exit(-1);
    }
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, gpu_device) != cudaSuccess || cudaSetDevice(gpu_device) != cudaSuccess) die("GPUDeviceInfo");
    printf("device %d: %s, compute capability %d.%d, %d SMs, %.1f GB global memory, %.1f MB L2, %zu KB shared memory "
           "per block (opt-in), clock %.0f MHz\n",
           gpu_device, p.name, p.major, p.minor, p.multiProcessorCount, p.totalGlobalMem / 1e9, p.l2CacheSize / 1e6,
           p.sharedMemPerBlockOptin / 1024, p.clockRate / 1e3);
}

}  // extern "C"
