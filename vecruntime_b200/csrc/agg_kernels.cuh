// Launch-side declarations of the aggregate kernels (implemented in
// agg_kernels.cu), used by the C ABI layer (abi.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "agg_types.h"

namespace vr {

// Prebuilt aggregate kernel variants (agg_aot_*.cu).
#define VR_AOT_DECL(name)                                                                                     \
    cudaError_t aot_launch_##name(const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter, \
                                  cudaStream_t stream);                                                      \
    int aot_regs_##name();
VR_AOT_DECL(direct)
VR_AOT_DECL(hash1)
VR_AOT_DECL(hash2)
VR_AOT_DECL(hash3)
VR_AOT_DECL(hash4)
#undef VR_AOT_DECL

SmemMap smem_map(int stages, int stage_bytes, int tier_bytes);

// Launchers (all asynchronous on `stream`). `descs` lives in device memory.
cudaError_t launch_aggregate(int kw, int tier, const BatchDesc* descs, const LaunchCfg& cfg, int blocks,
                             uint64_t* tile_counter, cudaStream_t stream);
// Registers per thread of the ahead-of-time aggregate kernel (occupancy).
int aggregate_kernel_regs(int kw, int tier);
// Replays deferred rows of one batch against the HBM table (no shared tier).
cudaError_t launch_replay(int kw, const BatchDesc* desc, const int64_t* rows, int64_t n, int g_probes,
                          cudaStream_t stream);
// Merges `n` slot states (stride sw words) into the table of `desc`
// (rehash into a larger table, spilled shared-tier slots).
cudaError_t launch_merge_slots(int kw, const BatchDesc* desc, const uint64_t* slots, int64_t n,
                               int g_probes, cudaStream_t stream);
// Compaction: out[i] = slot index of the i-th occupied slot; count in *num_dev.
// With temp == nullptr only sizes the scratch (*temp_bytes).
cudaError_t launch_compact_kw(int kw, const uint64_t* table, int64_t slots, int sw, int64_t* out, int64_t* num_dev,
                              void* temp, size_t* temp_bytes, cudaStream_t stream);
// Uploads the 10^p table used by the decimal precision checks (per device).
// Writes output rows [from, to) of the compacted groups into device columns.
cudaError_t launch_emit(const Program* prog_dev, const EmitProgram* emit_dev, const uint64_t* table,
                        const int64_t* slot_of, int64_t from, int64_t to, const vr_out_column* outs_dev,
                        uint64_t* ctrl, cudaStream_t stream);
// One key column of the row hash, as the kernel reads it.
struct HashKey {
    const void* data;
    const uint8_t* validity;      // nullptr: every row valid
    const int32_t* offsets;       // VR_UTF8: n + 1 offsets into data
    const uint32_t* dict_hashes;  // VR_DICT32: hashBytes of each dictionary entry
    int32_t lane;
    int32_t dict_size;            // VR_DICT32: entries; an id outside [0, dict_size) mixes 0
};
static_assert(sizeof(HashKey) == 40, "HashKey layout");
// vr_hash_rows_noalloc's fixed scratch: at most this many key descriptors.
constexpr int kHashRowsScratchMaxKeys = 16;
constexpr size_t kHashRowsScratchBytes = kHashRowsScratchMaxKeys * sizeof(HashKey);
static_assert(kHashRowsScratchBytes == 640, "the header documents a 640-byte scratch");
// The scratch's device address on the current device.
cudaError_t hash_rows_scratch_address(void** out);

// Reference row hash (HashKernels.java) over device key columns; `bad_id`
// (optional) receives 1 when a dictionary id lies outside its dictionary.
cudaError_t launch_hash_rows(int num_keys, const HashKey* keys_dev, int64_t n, uint32_t* out, int finish,
                             uint32_t* bad_id, cudaStream_t stream);
// HashKernels.hashBytes of every entry of a device dictionary (NULL_MARK for a null entry).
cudaError_t launch_hash_dictionary(const vr_dictionary& dict, uint32_t* out, cudaStream_t stream);

}  // namespace vr
