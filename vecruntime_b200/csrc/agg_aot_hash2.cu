// Prebuilt aggregate kernel, variant hash2 (key width 2, kTierHash).
#include "agg_aot.cuh"

namespace vr {
cudaError_t aot_launch_hash2(const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                          cudaStream_t stream) {
    return aot_launch<2, kTierHash>(descs, cfg, blocks, tile_counter, stream);
}
int aot_regs_hash2() { return aot_regs<2, kTierHash>(); }
}  // namespace vr
