// capi.cu -- extern "C" surface of librhmc_b200 (declared in include/rhmc_b200.h):
// context lifecycle, field I/O and the Dslash entry points.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "capi_util.h"
#include "context.h"
#include "kernels.h"

namespace rhmc {

static thread_local std::string g_err;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(RHMC_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Copies a caller buffer to the device if it lives on the host; returns the device pointer.
int stage_in(rhmc_ctx *c, const char *slot, const void *src, size_t bytes, int location, const void **dev)
{
    if (location == RHMC_DEVICE) { *dev = src; return RHMC_OK; }
    if (location != RHMC_HOST) return fail(RHMC_ERR_ARG, "location must be RHMC_HOST or RHMC_DEVICE");
    void *p;
    CK(c->ws.get(slot, bytes, &p));
    CK(cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, c->stream));
    *dev = p;
    return RHMC_OK;
}

}  // namespace rhmc

using namespace rhmc;

extern "C" {

const char *rhmc_last_error(void) { return g_err.c_str(); }

int rhmc_create(const rhmc_params *p, rhmc_ctx **out)
{
    if (!p || !out) return fail(RHMC_ERR_ARG, "null argument");
    *out = nullptr;
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->nt <= 0 || (p->nx | p->ny | p->nz | p->nt) & 1)
        return fail(RHMC_ERR_ARG, "lattice extents must be positive and even (got %d %d %d %d)", p->nx, p->ny, p->nz, p->nt);
    const long V = (long)p->nx * p->ny * p->nz * p->nt;
    if (V / 2 > 0x3fffffffL) return fail(RHMC_ERR_ARG, "lattice too large for 32-bit site indices");
    CK(cudaSetDevice(p->device));
    rhmc_ctx *c = new rhmc_ctx();
    c->g.nx = p->nx; c->g.ny = p->ny; c->g.nz = p->nz; c->g.nt = p->nt;
    c->g.Vh = (int)(V / 2);
    c->g.antiperiodic_t = p->ferm_temp_bc == 0;
    geom_divisors(c->g);
    c->V = V; c->Vh = V / 2;
    c->device = p->device;
    c->mass = p->mass;
    c->beta = p->beta;
    c->U64 = nullptr; c->U64_12 = nullptr; c->U32_18 = nullptr; c->U32_12 = nullptr; c->U16_12 = nullptr;
    c->P = nullptr; c->IP = nullptr;
    for (int i = 0; i < 5; i++) c->derived_valid[i] = false;
    c->launches = 0;
    c->hflags = nullptr;
    c->driver = nullptr;
    c->dh_ready = false;
    c->dh_cmp = c->dh_down = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&c->hflags, 256, cudaHostAllocDefault);
    c->aux = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    c->own_stream = true;
    if (e == cudaSuccess) e = cudaMalloc(&c->U64, 8 * 9 * c->Vh * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&c->P, 8 * 8 * c->Vh * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&c->IP, 8 * 8 * c->Vh * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(c->U64, 0, 8 * 9 * c->Vh * sizeof(double2), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->P, 0, 8 * 8 * c->Vh * sizeof(double), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->IP, 0, 8 * 8 * c->Vh * sizeof(double), c->stream);
    if (e != cudaSuccess) {
        rhmc_destroy(c);
        return cuda_fail(e, "rhmc_create");
    }
    *out = c;
    return RHMC_OK;
}

int rhmc_destroy(rhmc_ctx *c)
{
    if (!c) return RHMC_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->U64); cudaFree(c->U64_12); cudaFree(c->U32_18); cudaFree(c->U32_12); cudaFree(c->U16_12);
    cudaFree(c->P); cudaFree(c->IP);
    c->graphs.release();
    c->ws.release();
    driver_free(c->driver);
    if (c->hflags) cudaFreeHost(c->hflags);
    if (c->aux) {
        cudaStreamDestroy(c->aux);
        cudaEventDestroy(c->ev_fork);
        cudaEventDestroy(c->ev_join);
    }
    if (c->dh_ready) {
        cudaStreamDestroy(c->dh_cmp);
        cudaStreamDestroy(c->dh_down);
        for (int i = 0; i < RHMC_DH_MAXCH; i++) {
            cudaEventDestroy(c->dh_up_ev[i]);
            cudaEventDestroy(c->dh_cmp_ev[i]);
        }
        cudaEventDestroy(c->dh_done);
    }
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return RHMC_OK;
}

int rhmc_set_stream(rhmc_ctx *c, void *stream)
{
    if (!c) return fail(RHMC_ERR_ARG, "null context");
    if (stream) {
        if (c->own_stream) { cudaStreamSynchronize(c->stream); cudaStreamDestroy(c->stream); }
        c->stream = (cudaStream_t)stream;
        c->own_stream = false;
    } else if (!c->own_stream) {
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    return RHMC_OK;
}

int rhmc_sync(rhmc_ctx *c)
{
    if (!c) return fail(RHMC_ERR_ARG, "null context");
    CK(cudaStreamSynchronize(c->stream));
    return RHMC_OK;
}

int rhmc_launch_count(const rhmc_ctx *c, long *count)
{
    if (!c || !count) return fail(RHMC_ERR_ARG, "null argument");
    *count = c->launches;
    return RHMC_OK;
}

int rhmc_geometry(rhmc_ctx *c, int *table, int *eta)
{
    if (!c) return fail(RHMC_ERR_ARG, "null context");
    void *dt = nullptr, *de = nullptr;
    if (table) CK(c->ws.get("geom_table", 8 * c->V * sizeof(int), &dt));
    if (eta) CK(c->ws.get("geom_eta", 4 * c->V * sizeof(int), &de));
    launch_geometry(c, (int *)dt, (int *)de);
    CK(cudaGetLastError());
    if (table) CK(cudaMemcpyAsync(table, dt, 8 * c->V * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    if (eta) CK(cudaMemcpyAsync(eta, de, 4 * c->V * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return RHMC_OK;
}

int rhmc_set_gauge(rhmc_ctx *c, const double *u, int location)
{
    if (!c || !u) return fail(RHMC_ERR_ARG, "null argument");
    const void *d;
    int s = stage_in(c, "stage_gauge", u, 4 * c->V * 18 * sizeof(double), location, &d);
    if (s) return s;
    launch_gauge_from_ref(c, (const double *)d);
    invalidate_links(c);
    CK(cudaGetLastError());
    return RHMC_OK;
}

int rhmc_get_gauge(rhmc_ctx *c, double *u, int location)
{
    if (!c || !u) return fail(RHMC_ERR_ARG, "null argument");
    const size_t bytes = 4 * c->V * 18 * sizeof(double);
    void *d = u;
    if (location == RHMC_HOST) CK(c->ws.get("stage_gauge", bytes, &d));
    launch_gauge_to_ref(c, (double *)d);
    CK(cudaGetLastError());
    if (location == RHMC_HOST) {
        CK(cudaMemcpyAsync(u, d, bytes, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return RHMC_OK;
}

static int set_algebra(rhmc_ctx *c, double *A, const double *m, int location, int antiherm)
{
    if (!c || !m) return fail(RHMC_ERR_ARG, "null argument");
    const void *d;
    int s = stage_in(c, "stage_alg", m, 4 * c->V * 18 * sizeof(double), location, &d);
    if (s) return s;
    launch_algebra_from_ref(c, A, (const double *)d, antiherm);
    CK(cudaGetLastError());
    return RHMC_OK;
}

static int get_algebra(rhmc_ctx *c, const double *A, double *m, int location, int antiherm)
{
    if (!c || !m) return fail(RHMC_ERR_ARG, "null argument");
    const size_t bytes = 4 * c->V * 18 * sizeof(double);
    void *d = m;
    if (location == RHMC_HOST) CK(c->ws.get("stage_alg", bytes, &d));
    launch_algebra_to_ref(c, (double *)d, A, antiherm);
    CK(cudaGetLastError());
    if (location == RHMC_HOST) {
        CK(cudaMemcpyAsync(m, d, bytes, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return RHMC_OK;
}

int rhmc_set_momenta(rhmc_ctx *c, const double *p, int location) { return set_algebra(c, c ? c->P : nullptr, p, location, 0); }
int rhmc_get_momenta(rhmc_ctx *c, double *p, int location) { return get_algebra(c, c ? c->P : nullptr, p, location, 0); }
int rhmc_set_ipdot(rhmc_ctx *c, const double *p, int location) { return set_algebra(c, c ? c->IP : nullptr, p, location, 1); }
int rhmc_get_ipdot(rhmc_ctx *c, double *p, int location) { return get_algebra(c, c ? c->IP : nullptr, p, location, 1); }

int rhmc_spinor_to_internal(rhmc_ctx *c, int fmt, void *internal, const double *ref, int n, int location)
{
    if (!c || !internal || !ref || n <= 0 || fmt < 0 || fmt > RHMC_LINKS_F16_12) return fail(RHMC_ERR_ARG, "bad argument");
    const void *d;
    int s = stage_in(c, "stage_spinor", ref, (size_t)n * c->Vh * 6 * sizeof(double), location, &d);
    if (s) return s;
    launch_spinor_to_internal(c, fmt, internal, (const double *)d, n);
    CK(cudaGetLastError());
    return RHMC_OK;
}

int rhmc_spinor_from_internal(rhmc_ctx *c, int fmt, double *ref, const void *internal, int n, int location)
{
    if (!c || !internal || !ref || n <= 0 || fmt < 0 || fmt > RHMC_LINKS_F16_12) return fail(RHMC_ERR_ARG, "bad argument");
    const size_t bytes = (size_t)n * c->Vh * 6 * sizeof(double);
    void *d = ref;
    if (location == RHMC_HOST) CK(c->ws.get("stage_spinor_out", bytes, &d));
    launch_spinor_from_internal(c, fmt, (double *)d, internal, n);
    CK(cudaGetLastError());
    if (location == RHMC_HOST) {
        CK(cudaMemcpyAsync(ref, d, bytes, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return RHMC_OK;
}

int rhmc_dslash(rhmc_ctx *c, int fmt, int parity_out, void *out, const void *in, int n)
{
    if (!c || !out || !in || n <= 0 || (parity_out != 0 && parity_out != 1) || fmt < 0 || fmt > RHMC_LINKS_F16_12)
        return fail(RHMC_ERR_ARG, "bad argument");
    cudaError_t e = launch_dslash(c, fmt, parity_out, out, in, spinor_stride(fmt, c->Vh), n, nullptr, 0.0, 0.5, nullptr, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "rhmc_dslash");
    return RHMC_OK;
}

int rhmc_dslash_repeat(rhmc_ctx *c, int fmt, void *even, void *odd, int n, int repeats)
{
    if (!c || !even || !odd || n <= 0 || repeats < 0 || fmt < 0 || fmt > RHMC_LINKS_F16_12) return fail(RHMC_ERR_ARG, "bad argument");
    const size_t stride = spinor_stride(fmt, c->Vh);
    for (int r = 0; r < repeats; r++) {
        cudaError_t e = launch_dslash(c, fmt, 1, odd, even, stride, n, nullptr, 0.0, 0.5, nullptr, nullptr);
        if (e == cudaSuccess) e = launch_dslash(c, fmt, 0, even, odd, stride, n, nullptr, 0.0, 0.5, nullptr, nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "rhmc_dslash_repeat");
    }
    return RHMC_OK;
}

}  // extern "C"

// The device address of host range [p, p + bytes) when it is page-locked memory mapped for the
// device at both ends (cudaHostAlloc / cudaHostRegister, any runtime of the process), else null.
static void *mapped_host(void *p, size_t bytes)
{
    cudaPointerAttributes a0, a1;
    if (cudaPointerGetAttributes(&a0, p) != cudaSuccess || cudaPointerGetAttributes(&a1, (char *)p + bytes - 1) != cudaSuccess) {
        cudaGetLastError();  // clear the sticky-free error of an unregistered pointer
        return nullptr;
    }
    if (a0.type != cudaMemoryTypeHost || a1.type != cudaMemoryTypeHost || !a0.devicePointer || !a1.devicePointer) return nullptr;
    if ((char *)a1.devicePointer - (char *)a0.devicePointer != (ptrdiff_t)(bytes - 1)) return nullptr;
    return a0.devicePointer;
}

extern "C" {

int rhmc_dslash_sites(rhmc_ctx *c, int parity_out, double *out, const double *in, long k_lo, long k_count)
{
    if (!c || !out || !in || (parity_out != 0 && parity_out != 1)) return fail(RHMC_ERR_ARG, "bad argument");
    if (k_lo < 0 || k_count < 1 || k_lo + k_count > c->Vh)
        return fail(RHMC_ERR_ARG, "rhmc_dslash_sites: sites [%ld, %ld) outside [0, %ld)", k_lo, k_lo + k_count, c->Vh);
    cudaError_t e = launch_dslash_f64_range(c, c->stream, parity_out, out, in, (int)k_lo, (int)k_count);
    if (e != cudaSuccess) return cuda_fail(e, "rhmc_dslash_sites");
    return RHMC_OK;
}

int rhmc_dslash_host(rhmc_ctx *c, int parity_out, double *out, const double *in)
{
    if (!c || !out || !in || (parity_out != 0 && parity_out != 1)) return fail(RHMC_ERR_ARG, "bad argument");
    const size_t bytes = (size_t)c->Vh * 6 * sizeof(double);
    void *din, *dout;  // device copies in the host layout
    CK(c->ws.get("dh_in", bytes, &din));
    CK(c->ws.get("dh_out", bytes, &dout));
    // Chunks of whole t-slabs (half index k runs t-slowest, so a slab is a contiguous range of k
    // and of the host array): the output of chunk j needs the input of chunks j-1, j, j+1.
    int nch = 0;
    for (int n = RHMC_DH_MAXCH; n >= 3; n--)
        if (c->g.nt % n == 0) { nch = n; break; }
    if (nch == 0) {  // too few time slices to pipeline: upload, Dslash, download
        CK(cudaMemcpyAsync(din, in, bytes, cudaMemcpyHostToDevice, c->stream));
        CK(launch_dslash_f64_range(c, c->stream, parity_out, dout, din, 0, (int)c->Vh));
        CK(cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return RHMC_OK;
    }
    if (!c->dh_ready) {
        // all or nothing: on a failure the handles made so far are released again
        cudaStream_t st[2] = {nullptr, nullptr};
        cudaEvent_t ev[2 * RHMC_DH_MAXCH + 1] = {};
        cudaError_t e = cudaStreamCreateWithFlags(&st[0], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st[1], cudaStreamNonBlocking);
        for (int i = 0; i < 2 * RHMC_DH_MAXCH + 1 && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            for (cudaStream_t s : st)
                if (s) cudaStreamDestroy(s);
            for (cudaEvent_t v : ev)
                if (v) cudaEventDestroy(v);
            return cuda_fail(e, "rhmc_dslash_host streams");
        }
        c->dh_cmp = st[0];
        c->dh_down = st[1];
        for (int i = 0; i < RHMC_DH_MAXCH; i++) {
            c->dh_up_ev[i] = ev[i];
            c->dh_cmp_ev[i] = ev[RHMC_DH_MAXCH + i];
        }
        c->dh_done = ev[2 * RHMC_DH_MAXCH];
        c->dh_ready = true;
    }
    // The library stream uploads chunk by chunk; the compute stream runs the Dslash of chunk j
    // once chunk j+1 is in.  When `out` is page-locked host memory (both ends of the range mapped
    // for the device), the Dslash stores each finished chunk straight into it over PCIe;
    // otherwise the download stream copies each finished chunk out.  Chunks 0 and nch-1 wrap
    // around in t, so they are computed last.  Uploads and the output traffic use opposite PCIe
    // directions and overlap each other and the kernels.
    const long cs = c->Vh / nch;  // sites per chunk
    const size_t cb = (size_t)cs * 6 * sizeof(double);
    double2 *hin = (double2 *)din, *hout = (double2 *)dout;
    double2 *zout = (double2 *)mapped_host(out, bytes);  // device address of out, or null
    auto upload = [&](int i) -> int {
        CK(cudaMemcpyAsync(hin + (size_t)i * cs * 3, in + (size_t)i * cs * 6, cb, cudaMemcpyHostToDevice, c->stream));
        CK(cudaEventRecord(c->dh_up_ev[i], c->stream));
        return RHMC_OK;
    };
    // the Dslash reads and writes the host layout directly (no conversion kernels)
    auto compute = [&](int j, int wait_for) -> int {
        CK(cudaStreamWaitEvent(c->dh_cmp, c->dh_up_ev[wait_for], 0));
        if (zout) {
            CK(launch_dslash_f64_range(c, c->dh_cmp, parity_out, zout, hin, (int)(j * cs), (int)cs));
            return RHMC_OK;
        }
        CK(launch_dslash_f64_range(c, c->dh_cmp, parity_out, hout, hin, (int)(j * cs), (int)cs));
        CK(cudaEventRecord(c->dh_cmp_ev[j], c->dh_cmp));
        CK(cudaStreamWaitEvent(c->dh_down, c->dh_cmp_ev[j], 0));
        CK(cudaMemcpyAsync(out + (size_t)j * cs * 6, hout + (size_t)j * cs * 3, cb, cudaMemcpyDeviceToHost, c->dh_down));
        return RHMC_OK;
    };
    int rc;
    for (int i = 0; i < nch; i++) {
        if ((rc = upload(i))) return rc;
        if (i >= 2 && (rc = compute(i - 1, i))) return rc;  // chunk i-1 needs chunks i-2 .. i
    }
    // the wrapping chunks: nch-1 needs 0 and nch-2; 0 needs nch-1 and 1 (all uploaded by now)
    if ((rc = compute(nch - 1, nch - 1)) || (rc = compute(0, nch - 1))) return rc;
    CK(cudaEventRecord(c->dh_done, zout ? c->dh_cmp : c->dh_down));
    CK(cudaStreamWaitEvent(c->stream, c->dh_done, 0));
    CK(cudaStreamSynchronize(c->stream));
    return RHMC_OK;
}

int rhmc_mdagm(rhmc_ctx *c, int fmt, void *out, const void *in, double shift, int n)
{
    if (!c || !out || !in || n <= 0 || fmt < 0 || fmt > RHMC_LINKS_F16_12) return fail(RHMC_ERR_ARG, "bad argument");
    const size_t st = spinor_stride(fmt, c->Vh);
    void *h;
    CK(c->ws.get("mdagm_h", (size_t)n * st * spinor_elem_bytes(fmt), &h));
    cudaError_t e = launch_dslash(c, fmt, 1, h, in, st, n, nullptr, 0.0, 0.5, nullptr, nullptr);
    if (e == cudaSuccess) e = launch_dslash(c, fmt, 0, out, h, st, n, in, c->mass * c->mass + shift, -0.5, nullptr, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "rhmc_mdagm");
    return RHMC_OK;
}

}  // extern "C"
