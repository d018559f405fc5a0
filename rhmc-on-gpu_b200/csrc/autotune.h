// autotune.h -- runtime choice of launch configurations (no counterpart in the reference, which
// fixes 128 threads per block for every kernel, include/global_macro.h:8).
//
// Every Dslash instantiation is compiled in three launch shapes (threads per block, minimum
// resident blocks per SM); shape 0 is the compiled-in default of DslashCfg.  The first time an
// instantiation runs on a device at a volume (outside a stream capture), each shape is timed
// with CUDA events on scratch spinors and the fastest is recorded; later launches, including the
// ones captured into the solvers' graphs, use it.  The batched host-side Dslash (n right-hand
// sides that no single instantiation carries) likewise times its RHS packings (splitting n into
// launches of at most 8, 4 or 3 right-hand sides).  Choices are keyed by the device's name, the
// volume and the kernel, kept for the process, and optionally read from and written to a JSON
// cache file (RHMC_TUNE_CACHE, or rhmc_tune_cache_load/_save).
//
// Launch shapes only change the grid and the register budget, never the arithmetic: outputs,
// including the block-size-independent reductions, are bit-identical whichever shape runs.
#pragma once
#include <cuda_runtime.h>
#include <string>

namespace rhmc {

struct DsShape {
    int block, minb;
};

// process-wide switch (default on; RHMC_AUTOTUNE=0 in the environment turns it off)
bool autotune_enabled();
// < 0: tuned choices; >= 0: every tuned launch uses that candidate index (tests, diagnostics)
int autotune_override();
// the chosen candidate for key, or -1 when it has not been tuned yet (loads the cache file on
// first use)
int tune_get(const std::string &key);
// records a choice and the candidates' times (microseconds); saves the cache file when one is set
void tune_put(const std::string &key, int choice, const float *us, const DsShape *shapes, int n);
// "<device name>|vh=<Vh>|<what>"
std::string tune_key(long vh, const std::string &what);
// true when stream s is capturing (nothing may be timed on it then)
bool stream_capturing(cudaStream_t s);
// Grid for a kernel that walks ntiles tiles of `block` threads with stride gridDim.x: one wave of
// persistent blocks (SMs x resident blocks of that kernel on the current device, queried once
// per device and kernel), or ntiles when that is smaller or unknown.
int persistent_grid(const void *kern, int block, int ntiles);

}  // namespace rhmc
