// The prebuilt (ahead-of-time) aggregate kernel: the same body as the
// per-spec kernels compiled at run time, with the Program read from global
// memory. Each agg_aot_*.cu instantiates one (key width, tier) variant so the
// variants compile in parallel.
#pragma once
#include "agg_device.cuh"
#include "agg_kernels.cuh"
#include "agg_main.cuh"

namespace vr {

template <int KW, int TIER>
__global__ void __launch_bounds__(kMaxConsumerThreads + 32, 1) k_aggregate(const BatchDesc* __restrict__ descs,
                                                                        const LaunchCfg cfg,
                                                                        uint64_t* __restrict__ tile_counter) {
    extern __shared__ __align__(128) unsigned char smem[];
    aggregate_body<KW, TIER>(descs, cfg, tile_counter, smem);
}

template <int KW, int TIER>
cudaError_t aot_launch(const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                       cudaStream_t stream) {
    auto fn = k_aggregate<KW, TIER>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, cfg.smem_bytes);
    if (e != cudaSuccess) return e;
    fn<<<blocks, cfg.consumer_threads + 32, cfg.smem_bytes, stream>>>(descs, cfg, tile_counter);
    return cudaGetLastError();
}

template <int KW, int TIER>
int aot_regs() {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, k_aggregate<KW, TIER>) != cudaSuccess) return 0;
    return a.numRegs;
}

}  // namespace vr
