// Launch-time types of the aggregate kernel, shared by the host runtime, the
// ahead-of-time kernels and the per-spec kernels compiled at run time (NVRTC):
// no host headers here.
#pragma once
#include "vr_internal.h"

namespace vr {

// Where each staged column lands inside one pipeline stage.
struct StageLayout {
    int32_t data_off[kMaxCols];
    int32_t valid_off[kMaxCols];  // -1: the column is never nullable
    int32_t sel_off;              // -1: launches without selection bitmaps
    int32_t stage_bytes;
};

struct LaunchCfg {
    int32_t tile_rows;         // rows per tile, a multiple of 128
    int32_t stages;            // pipeline depth
    int32_t consumer_threads;  // multiple of 32; one extra producer warp follows
    int32_t num_desc;          // instances in this launch
    int64_t total_tiles;
    int32_t g_probes;          // HBM table probe limit before a row is deferred
    int32_t s_probes;          // unused: the probe limit is per instance (BatchDesc::s_probes)
    int32_t smem_bytes;        // dynamic shared memory of the launch
    int32_t tier_bytes;        // shared memory of the tier area
    int32_t rchunk;            // rows per consumer thread per chunk: 2, 4 or 8 (direct), 1 (hash)
    int32_t wait_polls;        // bounded barrier waits: suspended polls of up to 1 ms before giving up
    int32_t test_stall;        // test hook: the producer leaves at once, so consumer waits run out
    int32_t tile_run;          // tiles a producer takes per grab from the work counter (1 or more):
                               // consecutive tiles, so fewer CTAs touch each small instance
    StageLayout lay;
};

// Shared-memory map of the aggregate kernel (same formula on host and device).
struct SmemMap {
    int32_t prog, desc, pdesc, bars, hdr, stages, tier, total;
};

constexpr int kMaxStages = 4;
constexpr int kMaxConsumerThreads = 256;     // the prebuilt kernel's launch bounds
constexpr int kWholeTableThreads = 512;      // one CTA per SM holding a group table in shared memory
constexpr int kMaxConsumerThreadsJit = 992;  // per-spec kernels take their bounds from the shape (992 + the producer warp = 1,024)

}  // namespace vr
