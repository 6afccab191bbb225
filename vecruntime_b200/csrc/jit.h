// Per-spec aggregate kernels compiled at run time with NVRTC (see jit.cpp).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "agg_types.h"

namespace vr {

struct JitKernel;

// The kernel for (program, kw, tier) on `device`, compiling it on first use
// (cached per process, and on disk under $VRGPU_JIT_CACHE when set).
// Returns nullptr (with `err` set) when NVRTC or the driver is unavailable or
// the compile fails; callers then use the ahead-of-time kernel.
// What a per-spec kernel is compiled for besides the Program: key width,
// tier, rows per thread per chunk, and its launch bounds (consumer threads,
// CTAs per SM the register budget must allow).
struct JitShape {
    int kw = 1;
    int tier = 0;
    int rchunk = 4;
    int threads = 256;
    int min_blocks = 1;
    int warp_agg = 1;  // 0: no launch of this kernel pre-aggregates in the warp (the code is left out)
};
JitKernel* jit_get(const Program& prog, const JitShape& shape, int device, std::string* err);
int jit_regs(const JitKernel* k);
cudaError_t jit_launch(JitKernel* k, const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                       cudaStream_t stream);
// Whether per-spec compilation is enabled ($VRGPU_JIT != "0").
bool jit_enabled();
// Compiles (NVRTC only, no device needed) and reports the cubin size.
bool jit_compile_only(const Program& prog, const JitShape& shape, size_t* cubin_bytes, std::string* err);

}  // namespace vr
