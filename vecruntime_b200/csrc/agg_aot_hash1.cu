// Prebuilt aggregate kernel, variant hash1 (key width 1, kTierHash).
#include "agg_aot.cuh"

namespace vr {
cudaError_t aot_launch_hash1(const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                          cudaStream_t stream) {
    return aot_launch<1, kTierHash>(descs, cfg, blocks, tile_counter, stream);
}
int aot_regs_hash1() { return aot_regs<1, kTierHash>(); }
}  // namespace vr
