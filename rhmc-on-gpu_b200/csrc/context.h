// context.h -- the device-resident state behind one rhmc_ctx handle.
//
// The reference keeps its device state in file-scope globals that are reallocated every
// trajectory (lib/Cuda/cuda_rhmc.cuh:73-79, lib/Cuda/cuda_init.cu:5-109) and mallocs solver
// scratch on every call (lib/Cuda/cuda_inverter.cu:463,594).  Here every field lives in one
// context for the lifetime of the handle; scratch is a grow-only named workspace.
#pragma once
#include <cuda_runtime.h>
#include <map>
#include <string>
#include <vector>

#include "rhmc_core.cuh"
#include "../../include/rhmc_b200.h"

namespace rhmc {

struct Driver;

struct Workspace {
    std::map<std::string, std::pair<void *, size_t>> buf;
    cudaError_t get(const std::string &name, size_t bytes, void **out)
    {
        auto it = buf.find(name);
        if (it != buf.end() && it->second.second >= bytes) { *out = it->second.first; return cudaSuccess; }
        if (it != buf.end()) { cudaFree(it->second.first); buf.erase(it); }
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
        if (e != cudaSuccess) return e;
        buf[name] = std::make_pair(p, bytes);
        *out = p;
        return cudaSuccess;
    }
    void release()
    {
        for (auto &kv : buf) cudaFree(kv.second.first);
        buf.clear();
    }
};

// Instantiated CUDA graphs of the solver loops, keyed by everything their kernels capture
// (pointers, sizes, coefficients, stream), so that a solve repeated with the same buffers and
// shifts (every force evaluation of a trajectory) replays the graph without re-capturing and
// re-instantiating it.  Least recently used entries are destroyed beyond `cap`.
struct GraphCache {
    struct Entry {
        std::string key;
        cudaGraphExec_t exec;
        unsigned long used;
    };
    std::vector<Entry> e;
    unsigned long tick = 0;
    size_t cap = 48;
    cudaGraphExec_t find(const std::string &k)
    {
        for (Entry &x : e)
            if (x.key == k) {
                x.used = ++tick;
                return x.exec;
            }
        return nullptr;
    }
    void put(const std::string &k, cudaGraphExec_t g)
    {
        if (e.size() >= cap) {
            size_t lru = 0;
            for (size_t i = 1; i < e.size(); i++)
                if (e[i].used < e[lru].used) lru = i;
            cudaGraphExecDestroy(e[lru].exec);
            e.erase(e.begin() + lru);
        }
        e.push_back({k, g, ++tick});
    }
    void release()
    {
        for (Entry &x : e) cudaGraphExecDestroy(x.exec);
        e.clear();
    }
};

// the bytes of a plain-data key (zero-initialise the struct before filling it)
template <class K>
inline std::string key_bytes(const K &k) { return std::string(reinterpret_cast<const char *>(&k), sizeof(K)); }

}  // namespace rhmc

constexpr int RHMC_DH_MAXCH = 16;  // chunks of the pipelined host-buffer Dslash

struct rhmc_ctx {
    rhmc::Geom g;
    long V, Vh;
    int device;
    double mass, beta;
    cudaStream_t stream;
    bool own_stream;
    // gauge field: FP64 18-real master ([mu][parity][9][Vh] double2) + derived formats
    double2 *U64;
    double2 *U64_12;
    float4 *U32_18;
    float4 *U32_12;
    uint4 *U16_12;
    bool derived_valid[5];
    // momenta and ipdot: FP64 algebra planes [mu][parity][8][Vh]
    double *P;
    double *IP;
    rhmc::Workspace ws;
    int *hflags;   // pinned host words for polling device-side solver flags
    // graph-captured solver loops run on this stream, ordered against `stream` by events
    // (capture is not possible on the legacy default stream a caller may have installed)
    cudaStream_t aux;
    cudaEvent_t ev_fork, ev_join;
    long launches;  // kernels launched by this context (counted by the host wrappers)
    rhmc::GraphCache graphs;  // instantiated solver-loop graphs
    rhmc::Driver *driver;  // molecular-dynamics driver state (rhmc_driver_setup), or null
    // pipelined host-buffer Dslash: compute and download streams, per-chunk events (made on first use)
    cudaStream_t dh_cmp, dh_down;
    cudaEvent_t dh_up_ev[RHMC_DH_MAXCH], dh_cmp_ev[RHMC_DH_MAXCH], dh_done;
    bool dh_ready;
};

namespace rhmc {
// link format accessor for kernels; ensures the derived copy is current
cudaError_t links_f64_18(rhmc_ctx *c, L64_18 *lf);
cudaError_t links_f64_12(rhmc_ctx *c, L64_12 *lf);
cudaError_t links_f32_18(rhmc_ctx *c, L32_18 *lf);
cudaError_t links_f32_12(rhmc_ctx *c, L32_12 *lf);
cudaError_t links_f16_12(rhmc_ctx *c, L16_12 *lf);
// elements between consecutive spinors of a link format's internal storage (Vh 16-byte
// vectors for half, 3*Vh complex numbers otherwise)
inline size_t spinor_stride(int fmt, long Vh) { return (fmt == RHMC_LINKS_F16_12 ? 1 : 3) * (size_t)Vh; }
inline size_t spinor_elem_bytes(int fmt)
{
    return (fmt == RHMC_LINKS_F64_18 || fmt == RHMC_LINKS_F64_12 || fmt == RHMC_LINKS_F16_12) ? 16 : 8;
}
void invalidate_links(rhmc_ctx *c);
int grid_for(long n, int block);
void driver_free(Driver *d);

// Work issued on c->aux between the constructor and the destructor is ordered after
// everything already on c->stream and before anything issued on it later.
struct AuxScope {
    rhmc_ctx *c;
    explicit AuxScope(rhmc_ctx *cc) : c(cc)
    {
        cudaEventRecord(c->ev_fork, c->stream);
        cudaStreamWaitEvent(c->aux, c->ev_fork, 0);
    }
    ~AuxScope()
    {
        cudaEventRecord(c->ev_join, c->aux);
        cudaStreamWaitEvent(c->stream, c->ev_join, 0);
    }
};
}  // namespace rhmc
