// Prebuilt aggregate kernel, variant hash4 (key width 4, kTierHash).
#include "agg_aot.cuh"

namespace vr {
cudaError_t aot_launch_hash4(const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                          cudaStream_t stream) {
    return aot_launch<4, kTierHash>(descs, cfg, blocks, tile_counter, stream);
}
int aot_regs_hash4() { return aot_regs<4, kTierHash>(); }
}  // namespace vr
