// Prebuilt aggregate kernel, variant direct (key width 1, kTierDirect).
#include "agg_aot.cuh"

namespace vr {
cudaError_t aot_launch_direct(const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                          cudaStream_t stream) {
    return aot_launch<1, kTierDirect>(descs, cfg, blocks, tile_counter, stream);
}
int aot_regs_direct() { return aot_regs<1, kTierDirect>(); }
}  // namespace vr
