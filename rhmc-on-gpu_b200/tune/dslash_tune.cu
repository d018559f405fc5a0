// dslash_tune.cu -- offline sweep of the Dslash launch configurations (DslashCfg in
// csrc/dslash.cuh).  For the link formats and RHS counts the solvers launch, it times the
// half-Dslash kernel with and without the fused reductions for a set of (threads per block,
// minimum resident blocks per SM) pairs, with CUDA events over 20 back-to-back launches after 3
// warm-ups, and prints registers, spills, resident blocks and GB/s of algorithmic traffic.
// DslashCfg encodes the fastest pair of each case.  Inputs are deterministic patterns (the
// timing does not depend on the values).
//   make -C rhmc-on-gpu_b200 tune && rhmc-on-gpu_b200/_build/dslash_tune 32 32 [filter [shape [persist]]]
// filter: run only the cases whose "<format> NR=<n> red=<0|1>" label contains it; shape
// "<block>x<minb>": run only that launch shape (for a profiler capture; "all": every shape);
// persist 1: launch one wave of persistent blocks that walk the tiles instead of one block per
// tile.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "../csrc/dslash.cuh"
using namespace rhmc;

#define CKE(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { printf("CUDA %s at %d\n", cudaGetErrorString(e_), __LINE__); exit(1); } } while (0)

__global__ void fill(double *p, long n, double s) { long i = (long)blockIdx.x * blockDim.x + threadIdx.x; if (i < n) p[i] = s * (double)((i * 2654435761u) % 1000) / 1000.0 - 0.5 * s; }

static Geom G;
static void *Ubuf, *In, *Out, *Y, *Part;
static unsigned *Tick;
static cudaEvent_t e0, e1;
static const char *Filter = nullptr;
static const char *Only = nullptr;  // "<block>x<minb>": run only that launch shape
static int Persist = 0;             // 1: persistent grid
static int NSM = 148;

// RED: the solver's D_eo launch (y read, fused reduction); YONLY: y read without the reduction
template <class LF, int NR, bool RED, int B, int MB, bool YONLY = false>
void timeit(const char *lname, LF lf)
{
    typedef typename LF::real R;
    typedef typename LF::store::elem E;
    if (Only) {
        char shape[32];
        snprintf(shape, sizeof(shape), "%dx%d", B, MB);
        if (strcmp(shape, Only)) return;
    }
    DslashArgs<LF, NR, NoFin> a;
    memset(&a, 0, sizeof(a));
    a.g = G; a.p_out = 1; a.links = lf; a.in = (const E *)In; a.out = (E *)Out; a.y = (RED || YONLY) ? (const E *)Y : nullptr;
    a.stride = (size_t)LF::store::planes * G.Vh; a.alpha = (R)0.01; a.beta = (R)-0.5; a.use_alphas = 0;
    for (int r = 0; r < NR; r++) a.alphas[r] = (R)0.01;
    a.partials = (double *)Part; a.ticket = Tick;
    auto kern = dslash_kernel<LF, NR, RED || YONLY, RED, NoFin, B, MB>;
    const int ntiles = (int)(((long)G.Vh + B - 1) / B);
    cudaFuncAttributes fa;
    cudaFuncGetAttributes(&fa, kern);
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, B, 0);
    // one tile per block, or persistent blocks (one wave: SMs x resident blocks) walking the tiles
    const int grid = Persist ? (ntiles < NSM * nb ? ntiles : NSM * nb) : ntiles;
    for (int i = 0; i < 3; i++) {
        kern<<<grid, B>>>(a);
        CKE(cudaGetLastError());
    }
    CKE(cudaDeviceSynchronize());
    const int REP = 20;
    cudaEventRecord(e0);
    for (int i = 0; i < REP; i++) kern<<<grid, B>>>(a);
    cudaEventRecord(e1);
    CKE(cudaEventSynchronize(e1));
    float ms;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= REP;
    const double ws = LF::store::planes == 1 ? 16.0 / 6.0 : sizeof(typename LF::store::real);  // bytes per spinor real
    const double bytes = (double)G.Vh * (8.0 * LF::bytes + NR * (12.0 + ((RED || YONLY) ? 6.0 : 0.0)) * ws);
    printf("%-7s NR=%d red=%d y=%d block=%3d minb=%d grid=%5d regs=%3d spill=%4d blocks/SM=%d  %8.1f us  %7.1f GB/s\n",
           lname, NR, (int)RED, (int)(RED || YONLY), B, MB, grid, fa.numRegs, (int)fa.localSizeBytes, nb, ms * 1e3,
           bytes / (ms * 1e-3) / 1e9);
}

template <class LF, int NR, bool RED>
void sweep(const char *n, LF lf)
{
    char label[64];
    snprintf(label, sizeof(label), "%s NR=%d red=%d", n, NR, (int)RED);
    if (Filter && !strstr(label, Filter)) return;
    timeit<LF, NR, RED, 256, 1>(n, lf);
    timeit<LF, NR, RED, 256, 2>(n, lf);
    timeit<LF, NR, RED, 128, 2>(n, lf);
    timeit<LF, NR, RED, 128, 3>(n, lf);
    timeit<LF, NR, RED, 128, 4>(n, lf);
    timeit<LF, NR, RED, 128, 6>(n, lf);
    if constexpr (!RED) timeit<LF, NR, RED, 64, 8>(n, lf);  // the reductions need blocks of 128 or 256 threads
    // the y read alone, to separate its cost from the reduction's
    if constexpr (RED) {
        timeit<LF, NR, false, 128, 3, true>(n, lf);
        timeit<LF, NR, false, 128, 4, true>(n, lf);
        timeit<LF, NR, false, 256, 2, true>(n, lf);
    }
}

int main(int argc, char **argv)
{
    const int nx = argc > 1 ? atoi(argv[1]) : 32, nt = argc > 2 ? atoi(argv[2]) : 32;
    Filter = argc > 3 ? argv[3] : nullptr;
    Only = argc > 4 && strcmp(argv[4], "all") ? argv[4] : nullptr;
    Persist = argc > 5 ? atoi(argv[5]) : 0;
    cudaDeviceGetAttribute(&NSM, cudaDevAttrMultiProcessorCount, 0);
    G = Geom{nx, nx, nx, nt, nx * nx * nx * nt / 2, 1, {}, {}, {}};
    geom_divisors(G);
    const long Vh = G.Vh;
    printf("lattice %d^3x%d Vh=%ld\n", nx, nt, Vh);
    const size_t ub = (size_t)72 * Vh * 16, vb = (size_t)8 * 3 * Vh * 16;  // links FP64-18; 8 RHS FP64
    CKE(cudaMalloc(&Ubuf, ub));
    CKE(cudaMalloc(&In, vb));
    CKE(cudaMalloc(&Out, vb));
    CKE(cudaMalloc(&Y, vb));
    CKE(cudaMalloc(&Part, (size_t)(Vh / 64 + 1) * 16 * sizeof(double)));
    CKE(cudaMalloc(&Tick, 16));
    CKE(cudaMemset(Tick, 0, 16));
    fill<<<(ub / 8 + 255) / 256, 256>>>((double *)Ubuf, ub / 8, 1.0);
    fill<<<(vb / 8 + 255) / 256, 256>>>((double *)In, vb / 8, 1.0);
    fill<<<(vb / 8 + 255) / 256, 256>>>((double *)Y, vb / 8, 1.0);
    CKE(cudaDeviceSynchronize());
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    L64_18 l18; l18.p = (const double2 *)Ubuf; l18.Vh = (int)Vh;
    L64_12 l12; l12.p = (const double2 *)Ubuf; l12.Vh = (int)Vh;
    L32_12 f12; f12.p = (const float4 *)Ubuf; f12.Vh = (int)Vh;
    L32_18 f18; f18.p = (const float4 *)Ubuf; f18.Vh = (int)Vh;
    L16_12 h12; h12.p = (const uint4 *)Ubuf; h12.Vh = (int)Vh;
    sweep<L64_18, 1, false>("f64_18", l18);
    sweep<L64_18, 1, true>("f64_18", l18);
    sweep<L64_12, 1, false>("f64_12", l12);
    sweep<L64_12, 4, false>("f64_12", l12);
    sweep<L64_12, 4, true>("f64_12", l12);
    sweep<L64_18, 8, false>("f64_18", l18);
    sweep<L32_12, 1, false>("f32_12", f12);
    sweep<L32_12, 4, false>("f32_12", f12);
    sweep<L32_12, 4, true>("f32_12", f12);
    // the solvers' base vectors: right-hand sides packed 4 (FP32) or 2 (FP64) per 32-byte element
    LPack<L32_12, 4> f12q; f12q.p = f12.p; f12q.Vh = f12.Vh;
    LPack<L64_12, 2> l12p; l12p.p = l12.p; l12p.Vh = l12.Vh;
    sweep<LPack<L32_12, 4>, 4, false>("f32_12q", f12q);
    sweep<LPack<L32_12, 4>, 4, true>("f32_12q", f12q);
    sweep<LPack<L64_12, 2>, 4, false>("f64_12p", l12p);
    sweep<LPack<L64_12, 2>, 4, true>("f64_12p", l12p);
    sweep<L32_12, 8, false>("f32_12", f12);
    sweep<L32_12, 8, true>("f32_12", f12);
    sweep<L32_18, 1, false>("f32_18", f18);
    sweep<L16_12, 1, false>("f16_12", h12);
    sweep<L16_12, 8, false>("f16_12", h12);
    sweep<L16_12, 8, true>("f16_12", h12);
    CKE(cudaGetLastError());
    return 0;
}
