// Prebuilt aggregate kernel, variant hash3 (key width 3, kTierHash).
#include "agg_aot.cuh"

namespace vr {
cudaError_t aot_launch_hash3(const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                          cudaStream_t stream) {
    return aot_launch<3, kTierHash>(descs, cfg, blocks, tile_counter, stream);
}
int aot_regs_hash3() { return aot_regs<3, kTierHash>(); }
}  // namespace vr
