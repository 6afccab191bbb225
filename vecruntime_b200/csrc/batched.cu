// Batched aggregation: many independent instances (Spark tasks' batches of
// uneven row counts and cardinalities) in ONE persistent launch of
// k_aggregate. Tiles of every instance form one work space; CTAs pull tiles
// from a global counter, so a CTA that finishes a small instance moves on to
// the next tile of any instance. The whole step (table clears + the
// persistent launch) can be captured once as a CUDA graph and replayed.
//
// VR_BATCHED_PLAIN runs the same instances with one clear + one launch per
// instance, the baseline the persistent form is measured against.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "jit.h"
#include "runtime.h"

namespace vr {

struct ZeroSpan {
    uint64_t* ptr;
    int64_t words;
};

// Zeroes many buffers in one launch: block b takes span b % n with a stride.
__global__ void k_zero_many(const ZeroSpan* __restrict__ spans, int n) {
    for (int s = blockIdx.y; s < n; s += gridDim.y) {
        uint64_t* p = spans[s].ptr;
        const int64_t w = spans[s].words;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < w; i += (int64_t)gridDim.x * blockDim.x)
            p[i] = 0;
    }
}

// Gathers every instance's control block into one array (one D2H copy).
__global__ void k_gather_ctrl(const BatchDesc* __restrict__ descs, int n, uint64_t* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * CTRL_WORDS; i += gridDim.x * blockDim.x)
        out[i] = descs[i / CTRL_WORDS].ctrl[i % CTRL_WORDS];
}

}  // namespace vr

struct vr_batched {
    int device = 0;
    int mode = VR_BATCHED_PERSISTENT;
    bool use_graph = false;
    std::vector<vr_agg*> inst;
    std::vector<vr::BatchDesc> descs;
    vr::BatchDesc* descs_dev = nullptr;
    vr::ZeroSpan* spans_dev = nullptr;
    int num_spans = 0;
    uint64_t* counter = nullptr;
    uint64_t* ctrl_all_dev = nullptr;
    uint64_t* ctrl_all_host = nullptr;
    vr::LaunchCfg cfg{};  // the persistent launch: one block shape for every instance
    vr::JitKernel* jit = nullptr;
    int kw = 1, tier = vr::kTierHash, blocks = 0;
    int64_t total_tiles = 0;
    int64_t total_rows = 0;
    vr_batched_info info{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;  // the stream the graph was captured for
};

using namespace vr;

static cudaError_t persistent_launch(vr_batched* b, const LaunchCfg& L, cudaStream_t st) {
    if (b->jit) return jit_launch(b->jit, b->descs_dev, L, b->blocks, b->counter, st);
    return launch_aggregate(b->kw, b->tier, b->descs_dev, L, b->blocks, b->counter, st);
}

static int batched_enqueue(vr_batched* b, cudaStream_t st) {
    cudaError_t e;
    const int n = (int)b->inst.size();
    if (b->mode == VR_BATCHED_PERSISTENT) {
        dim3 grid(148 * 2, std::min(b->num_spans, 65535));
        k_zero_many<<<grid, 256, 0, st>>>(b->spans_dev, b->num_spans);
        if ((e = cudaGetLastError()) != cudaSuccess) return VR_ERR_CUDA;
        LaunchCfg L = b->cfg;
        L.total_tiles = b->total_tiles;
        L.num_desc = n;
        if ((e = persistent_launch(b, L, st)) != cudaSuccess) return VR_ERR_CUDA;
    } else {
        for (int i = 0; i < n; ++i) {
            vr_agg* h = b->inst[i];
            const BatchDesc& d = b->descs[i];
            if ((e = cudaMemsetAsync(h->table, 0, (size_t)h->table_slots * h->plan.prog.sw * 8, st)) != cudaSuccess)
                return VR_ERR_CUDA;
            if ((e = cudaMemsetAsync(d.ctrl, 0, CTRL_WORDS * 8, st)) != cudaSuccess) return VR_ERR_CUDA;
            LaunchCfg L = h->launch;
            L.total_tiles = d.num_tiles;
            int blocks = (int)std::min<int64_t>(h->blocks, d.num_tiles);
            if ((e = agg_launch(h, b->descs_dev + i, L, blocks, &d.ctrl[CTRL_NEXT_TILE], st)) != cudaSuccess)
                return VR_ERR_CUDA;
        }
    }
    k_gather_ctrl<<<(n * CTRL_WORDS + 255) / 256, 256, 0, st>>>(b->descs_dev, n, b->ctrl_all_dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return VR_ERR_CUDA;
    if ((e = cudaMemcpyAsync(b->ctrl_all_host, b->ctrl_all_dev, (size_t)n * CTRL_WORDS * 8, cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return VR_ERR_CUDA;
    return VR_OK;
}

// Rows a producer takes per grab in the persistent launch (a run of
// consecutive tiles of one instance), so a small instance is spread over
// fewer CTAs, each of which flushes its shared-memory table into the
// instance's HBM table. Measured on 512 uneven instances, 1,024-row tiles,
// 256 consumer threads: one tile per grab 23.1 ms, 4 tiles 21.4, 8 20.2, 16
// 19.2, 32 18.7, 128 19.8; with 512 consumer threads and the autotuner's
// strategies: 16,384 rows per grab 15.0 ms, 32,768 13.7, 65,536 13.2,
// 131,072 13.5.
constexpr int kBatchedRunRows = 65536;

// The persistent launch's block shape (hash tier): one for every instance,
// since the stage layout and the kernel's thread count are per launch.
// Measured defaults: two CTAs per SM of 512 consumer threads (the per-spec
// kernel fits them in 64 registers), 1,024-row tiles and two stages, which
// leave a 512-slot shared-memory area per CTA for 80-byte slots (a whole
// table for up to ~350 groups). On 512 uneven instances (tiles taken in runs,
// before / after the autotuner): 2 x 512 threads 13.9 / 12.4 ms, 2 x 384
// with 768-row tiles 14.9 / 13.6, 1 x 896 with 1,792-row tiles 14.8 / 13.4,
// 2 x 256 19.1 / 16.8, 2 x 480 with 512-row tiles 22.2 / 20.9.
static int batched_shape(vr_batched* b, const vr_tune_choice* shape) {
    vr_agg* h0 = b->inst[0];
    const Program& P = h0->plan.prog;
    const DeviceInfo& di = device_info(b->device);
    const int threads = shape && shape->threads ? shape->threads : 512;
    const int want_ctas = shape && shape->blocks_per_sm ? shape->blocks_per_sm : 2;
    const int T = shape && shape->tile_rows ? shape->tile_rows : 1024;
    if (threads % 32 || threads > kMaxConsumerThreadsJit || T % 128 || T <= 0) {
        set_thread_error("batched shape: threads must be a multiple of 32 up to 512, tiles a multiple of 128");
        return VR_ERR_INVALID;
    }
    const int budget = want_ctas <= 1 ? di.smem_optin : std::min(di.smem_optin, di.smem_per_sm / want_ctas - di.smem_reserved);
    const int stages = 2;
    const int sb = stage_bytes_for(P, T);
    const int base = smem_map(stages, sb, 0).total;
    if (base + 64 * 8 * P.sw > budget) {
        set_thread_error("batched shape: tiles too long for the shared memory of one block");
        return VR_ERR_UNSUPPORTED;
    }
    int64_t area = 1;
    while (area * 2 * 8 * P.sw <= budget - base) area *= 2;  // power-of-two tables
    LaunchCfg& L = b->cfg;
    L = h0->launch;
    L.tile_rows = T;
    L.tile_run = std::max(1, kBatchedRunRows / T);
    L.stages = stages;
    L.consumer_threads = threads;
    L.rchunk = 1;
    fill_layout(P, T, L.lay);
    L.tier_bytes = (int32_t)(area * 8 * P.sw);
    L.smem_bytes = smem_map(stages, sb, L.tier_bytes).total;
    b->info.smem_slots_max = (int32_t)area;
    // the spec's own kernel for this shape; the prebuilt one (up to 256 threads) otherwise
    int regs = aggregate_kernel_regs(b->kw, kTierHash);
    if (jit_enabled() && !(h0->spec.flags & VR_SPEC_NO_JIT)) {
        JitShape js;
        js.kw = P.kw;
        js.tier = kTierHash;
        js.rchunk = 1;
        js.threads = threads;
        js.min_blocks = ctas_per_sm(di, L.smem_bytes, 0, threads, want_ctas);
        js.warp_agg = 0;  // pre-aggregation compiled in only when an instance uses it
        for (vr_agg* h : b->inst) js.warp_agg |= h->cfg.warp_agg;
        std::string why;
        b->jit = jit_get(P, js, b->device, &why);
        if (b->jit) regs = jit_regs(b->jit);
    }
    if (!b->jit && threads > kMaxConsumerThreads) {
        set_thread_error("batched shape: more than 256 threads needs a per-spec kernel, which did not compile");
        return VR_ERR_UNSUPPORTED;
    }
    b->blocks = di.sms * ctas_per_sm(di, L.smem_bytes, regs, threads, want_ctas);
    return VR_OK;
}

// One instance's shared-memory strategy inside the persistent launch: its
// handle's own choice (the tuner's, else the default for its rows and
// estimated groups), fitted to the launch's shared-memory area.
//   whole table  -- every group in shared memory, probed until found: kept
//                   when the estimated groups fill at most 70% of a table
//                   that fits the area;
//   hot-key cache -- the first keys a CTA meets, two probes, then HBM;
//   HBM only     -- the handle chose no shared memory (tier 2).
static void instance_strategy(vr_batched* b, vr_agg* h, BatchDesc& d, int cache_slots) {
    const int64_t area = b->info.smem_slots_max;
    d.warp_agg = h->cfg.warp_agg;
    if (h->cfg.smem_slots <= 0) {
        d.smem_slots = 0;
        d.s_probes = 0;
        b->info.hbm_only++;
        return;
    }
    const int64_t est = h->spec.est_groups;
    if (h->cfg.s_probes > 2 && est > 0) {
        const int64_t need = next_pow2(std::max<int64_t>(64, (est * 10 + 6) / 7));
        if (need <= area) {
            d.smem_slots = (int32_t)need;
            d.s_probes = 64;
            b->info.whole_tables++;
            return;
        }
    }
    d.smem_slots = (int32_t)std::min<int64_t>(std::min<int64_t>(cache_slots, area), next_pow2(h->cfg.smem_slots));
    d.s_probes = 2;
    b->info.caches++;
}

static int batched_settle(vr_batched* b);

extern "C" {

int vr_batched_create(const vr_batched_plan* plan, vr_batched** out) {
    if (!plan || !out || plan->num_instances <= 0 || !plan->instances || !plan->batches) {
        set_thread_error("batched plan: null or empty");
        return VR_ERR_INVALID;
    }
    *out = nullptr;
    vr_batched* b = new vr_batched();
    b->mode = plan->mode;
    b->use_graph = plan->use_graph != 0;
    const int n = plan->num_instances;
    vr_agg* h0 = plan->instances[0];
    if (!h0) {
        delete b;
        set_thread_error("batched plan: null instance");
        return VR_ERR_INVALID;
    }
    b->device = h0->device;
    cudaSetDevice(b->device);
    // every instance shares the program (one kernel) and the tier
    for (int i = 0; i < n; ++i) {
        vr_agg* h = plan->instances[i];
        const vr_batch& bt = plan->batches[i];
        if (!h || h->dead || bt.location != VR_DEVICE) {
            delete b;
            set_thread_error("batched instances need live handles and device-resident batches");
            return VR_ERR_INVALID;
        }
        if (const char* why = batch_nullability_error(h, bt)) {
            delete b;
            set_thread_error(why);
            return VR_ERR_INVALID;
        }
        if (h->device != b->device || std::memcmp(&h->plan.prog, &h0->plan.prog, sizeof(Program)) != 0 ||
            h->cfg.tier != h0->cfg.tier) {
            delete b;
            set_thread_error("batched instances must share device, spec shape and tier");
            return VR_ERR_UNSUPPORTED;
        }
        if (h0->cfg.tier == kTierDirect && (h->cfg.tile_rows != h0->cfg.tile_rows || h->cfg.stages != h0->cfg.stages ||
                                            h->cfg.threads != h0->cfg.threads)) {
            delete b;
            set_thread_error("direct-tier batched instances must share their block shape");
            return VR_ERR_UNSUPPORTED;
        }
        if (!h->tdicts.empty()) {
            delete b;
            set_thread_error("batched launches take table-level dictionary ids, not batch dictionaries");
            return VR_ERR_UNSUPPORTED;
        }
        if (vr_agg_sync(h) != VR_OK) {
            delete b;
            set_thread_error("instance handle failed");
            return VR_ERR_STATE;
        }
        b->inst.push_back(h);
    }
    b->kw = h0->plan.prog.kw;
    b->tier = h0->cfg.tier;
    if (b->tier == kTierDirect) {
        b->cfg = h0->launch;
        b->jit = h0->jit;
        b->blocks = h0->blocks;
        b->info.smem_slots_max = 0;
    } else {
        int rc = batched_shape(b, plan->shape);
        if (rc != VR_OK) {
            delete b;
            return rc;
        }
    }
    b->info.jit = b->jit ? 1 : 0;
    const int cache_slots =
        plan->shape && plan->shape->smem_slots ? (int)next_pow2(plan->shape->smem_slots) : 256;
    // descriptors: instance i's tiles follow instance i-1's
    std::vector<ZeroSpan> spans;
    int64_t tile = 0;
    const int64_t T = b->mode == VR_BATCHED_PERSISTENT ? b->cfg.tile_rows : 0;
    for (int i = 0; i < n; ++i) {
        vr_agg* h = b->inst[i];
        const vr_batch& bt = plan->batches[i];
        StageSlot& s = h->slot[0];
        if (h->cfg.tier != kTierDirect && s.deferred_cap < bt.num_rows) {
            cudaFree(s.deferred);
            cudaFree(s.deferred_tmp);
            s.deferred_cap = std::max<int64_t>(bt.num_rows, 4096);
            if (cudaMalloc(&s.deferred, (size_t)s.deferred_cap * 8) != cudaSuccess ||
                cudaMalloc(&s.deferred_tmp, (size_t)s.deferred_cap * 8) != cudaSuccess) {
                vr_batched_destroy(b);
                set_thread_error("deferred-row lists: device memory");
                return VR_ERR_OOM;
            }
        }
        BatchDesc d;
        std::memset(&d, 0, sizeof(d));
        for (int c = 0; c < h->plan.prog.num_cols; ++c) {
            const vr_column& col = bt.columns[h->plan.spec_of_staged[c]];
            d.col_data[c] = (const char*)col.data;
            d.col_valid[c] = (const uint32_t*)col.validity;
        }
        d.selection = (const uint32_t*)bt.selection;
        fill_desc(h, bt, d, s.ctrl_dev, s, b->mode == VR_BATCHED_PERSISTENT ? tile : 0);
        if (T > 0) {  // the persistent launch's tiles and shared-memory strategy
            d.num_tiles = (bt.num_rows + T - 1) / T;
            if (b->tier != kTierDirect) instance_strategy(b, h, d, cache_slots);
        }
        bool tma = h->cfg.tma != 0;
        for (int c = 0; c < h->plan.prog.num_cols; ++c)
            tma = tma && ((uintptr_t)d.col_data[c] & 15) == 0 && ((uintptr_t)d.col_valid[c] & 15) == 0;
        d.tma = tma && ((uintptr_t)d.selection & 15) == 0;
        s.launched = d;
        b->descs.push_back(d);
        tile += d.num_tiles;
        b->total_rows += bt.num_rows;
        spans.push_back(ZeroSpan{h->table, h->table_slots * h->plan.prog.sw});
        spans.push_back(ZeroSpan{s.ctrl_dev, CTRL_WORDS});
        b->info.table_bytes += h->table_slots * h->plan.prog.sw * 8;
    }
    b->total_tiles = tile;
    b->info.threads = b->mode == VR_BATCHED_PERSISTENT ? b->cfg.consumer_threads : 0;
    b->info.tile_rows = b->mode == VR_BATCHED_PERSISTENT ? b->cfg.tile_rows : 0;
    b->info.stages = b->mode == VR_BATCHED_PERSISTENT ? b->cfg.stages : 0;
    b->info.blocks = b->mode == VR_BATCHED_PERSISTENT ? b->blocks : 0;
    b->info.smem_bytes = b->mode == VR_BATCHED_PERSISTENT ? b->cfg.smem_bytes : 0;
    b->info.total_tiles = tile;
    b->info.total_rows = b->total_rows;
    cudaError_t e;
    spans.push_back(ZeroSpan{nullptr, 0});
    b->num_spans = (int)spans.size() - 1;
    if ((e = cudaMalloc(&b->descs_dev, sizeof(BatchDesc) * n)) != cudaSuccess ||
        (e = cudaMalloc(&b->spans_dev, sizeof(ZeroSpan) * spans.size())) != cudaSuccess ||
        (e = cudaMalloc(&b->counter, 64)) != cudaSuccess ||
        (e = cudaMalloc(&b->ctrl_all_dev, (size_t)n * CTRL_WORDS * 8)) != cudaSuccess ||
        (e = cudaMallocHost(&b->ctrl_all_host, (size_t)n * CTRL_WORDS * 8)) != cudaSuccess) {
        vr_batched_destroy(b);
        set_thread_error("batched descriptors: device memory");
        return VR_ERR_OOM;
    }
    // the tile counter is zeroed with the tables
    b->num_spans += 1;
    spans[spans.size() - 1] = ZeroSpan{b->counter, 8};
    if ((e = cudaMemcpy(b->descs_dev, b->descs.data(), sizeof(BatchDesc) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(b->spans_dev, spans.data(), sizeof(ZeroSpan) * spans.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
        vr_batched_destroy(b);
        set_thread_error(std::string("batched descriptors: ") + cudaGetErrorString(e));
        return VR_ERR_CUDA;
    }
    *out = b;
    return VR_OK;
}

int vr_batched_get_info(const vr_batched* b, vr_batched_info* info) {
    if (!b || !info) return VR_ERR_INVALID;
    *info = b->info;
    return VR_OK;
}

int vr_batched_run(vr_batched* b, void* stream) {
    if (!b) return VR_ERR_INVALID;
    cudaSetDevice(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    int rc;
    // the launch zeros every table on `st`: a clear still queued on an
    // instance's own stream must not land in the middle of it
    for (vr_agg* h : b->inst) {
        if (!h->clear_queued) continue;
        if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return VR_ERR_CUDA;
        h->clear_queued = false;
    }
    if (b->use_graph) {
        if (!b->exec || b->graph_stream != st) {
            if (b->exec) cudaGraphExecDestroy(b->exec);
            if (b->graph) cudaGraphDestroy(b->graph);
            b->exec = nullptr;
            b->graph = nullptr;
            cudaStream_t cap = st;
            bool own = false;
            if (!cap) {  // the legacy stream cannot be captured
                cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
                own = true;
            }
            if ((e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return VR_ERR_CUDA;
            rc = batched_enqueue(b, cap);
            e = cudaStreamEndCapture(cap, &b->graph);
            if (own) cudaStreamDestroy(cap);
            if (rc != VR_OK || e != cudaSuccess) return VR_ERR_CUDA;
            if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) return VR_ERR_CUDA;
            b->graph_stream = st;
        }
        if ((e = cudaGraphLaunch(b->exec, st)) != cudaSuccess) return VR_ERR_CUDA;
    } else {
        rc = batched_enqueue(b, st);
        if (rc != VR_OK) return rc;
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return VR_ERR_CUDA;
    return batched_settle(b);
}

}  // extern "C"

// Per-instance bookkeeping after a run: groups, errors, and growth + replay
// where an instance's HBM table was too small.
static int batched_settle(vr_batched* b) {
    const int n = (int)b->inst.size();
    int status = VR_OK;
    for (int i = 0; i < n; ++i) {
        vr_agg* h = b->inst[i];
        StageSlot& s = h->slot[0];
        std::memcpy(s.ctrl_host, b->ctrl_all_host + (size_t)i * CTRL_WORDS, CTRL_WORDS * 8);
        h->groups_known = 0;
        h->compact_valid = false;
        h->stats.rows += b->descs[i].num_rows;
        h->stats.batches++;
        h->stats.kernel_launches++;
        s.launched = b->descs[i];
        s.pending = true;
        h->next_slot = 0;
        int64_t old_cap = h->cfg.capacity;
        int rc2 = agg_resolve_all(h);
        if (rc2 != VR_OK && status == VR_OK) status = rc2;
        if (h->cfg.capacity != old_cap) {  // grown: later runs use the new table
            BatchDesc d = b->descs[i];
            d.table = h->table;
            d.cap_mask = h->cfg.capacity - 1;
            b->descs[i] = d;
            cudaMemcpy(b->descs_dev + i, &d, sizeof(BatchDesc), cudaMemcpyHostToDevice);
            ZeroSpan zs{h->table, h->table_slots * h->plan.prog.sw};
            cudaMemcpy(b->spans_dev + 2 * i, &zs, sizeof(ZeroSpan), cudaMemcpyHostToDevice);
            // a captured graph reads the table pointers from these device
            // descriptors and spans, not from its kernel arguments: it stays valid
        }
    }
    return status;
}

// ---------------------------------------------------------------- autotuner
// Shared-memory strategies an instance can take in the persistent launch.
enum Strategy { kWhole = 0, kCache256, kCache512, kCache1024, kHbm, kStrategies };

// Sets instance d's strategy; false when it does not fit the launch's area.
static bool apply_strategy(const vr_batched* b, const vr_agg* h, BatchDesc& d, int s) {
    const int64_t area = b->info.smem_slots_max;
    switch (s) {
        case kWhole: {
            const int64_t est = h->spec.est_groups;
            if (est <= 0) return false;
            const int64_t need = next_pow2(std::max<int64_t>(64, (est * 10 + 6) / 7));
            if (need > area) return false;
            d.smem_slots = (int32_t)need;
            d.s_probes = 64;
            return true;
        }
        case kCache256:
        case kCache512:
        case kCache1024: {
            const int64_t slots = 256 << (s - kCache256);
            if (slots > area) return false;
            d.smem_slots = (int32_t)slots;
            d.s_probes = 2;
            return true;
        }
        case kHbm:
            d.smem_slots = 0;
            d.s_probes = 0;
            return true;
    }
    return false;
}

static int strategy_of(const BatchDesc& d) {
    if (d.smem_slots == 0) return kHbm;
    if (d.s_probes > 2) return kWhole;
    return d.smem_slots >= 1024 ? kCache1024 : d.smem_slots >= 512 ? kCache512 : kCache256;
}

// One timed persistent run (device time of the launch, then the bookkeeping).
static int timed_run(vr_batched* b, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, float* ms) {
    cudaEventRecord(e0, st);
    int rc = batched_enqueue(b, st);
    cudaEventRecord(e1, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return VR_ERR_CUDA;
    if (rc != VR_OK) return rc;
    cudaEventElapsedTime(ms, e0, e1);
    return batched_settle(b);
}

extern "C" {

int vr_batched_tune(vr_batched* b, int32_t iters, double* best_ms) {
    if (!b || b->mode != VR_BATCHED_PERSISTENT || b->tier == kTierDirect) {
        set_thread_error("vr_batched_tune: a persistent hash-tier launch only");
        return VR_ERR_INVALID;
    }
    if (iters < 1) iters = 2;
    cudaSetDevice(b->device);
    for (vr_agg* h : b->inst) {  // a clear still queued on an instance's own stream goes first
        if (!h->clear_queued) continue;
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) return VR_ERR_CUDA;
        h->clear_queued = false;
    }
    cudaStream_t st;
    cudaEvent_t e0, e1;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return VR_ERR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int n = (int)b->inst.size();
    auto upload = [&]() {
        return cudaMemcpy(b->descs_dev, b->descs.data(), sizeof(BatchDesc) * n, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    auto measure = [&](double* out) {
        double best = 1e30;
        for (int it = 0; it < iters + 1; ++it) {  // the first run warms up (and grows tables)
            float ms = 0;
            int rc = timed_run(b, st, e0, e1, &ms);
            if (rc != VR_OK) return rc;
            if (it > 0) best = std::min(best, (double)ms);
        }
        *out = best;
        return (int)VR_OK;
    };
    // instances grouped by the power of two of their estimated groups,
    // the buckets with the most rows tuned first
    std::map<int, std::vector<int>> buckets;
    std::map<int, int64_t> bucket_rows;
    for (int i = 0; i < n; ++i) {
        const int64_t est = std::max<int64_t>(1, b->inst[i]->spec.est_groups);
        int k = 0;
        while ((int64_t(1) << k) < est) ++k;
        buckets[k].push_back(i);
        bucket_rows[k] += b->descs[i].num_rows;
    }
    std::vector<std::pair<int64_t, int>> order;
    for (auto& kv : bucket_rows) order.push_back({-kv.second, kv.first});
    std::sort(order.begin(), order.end());
    double cur = 0;
    int rc = measure(&cur);
    // coordinate descent: each bucket's strategy with the others held fixed
    for (size_t oi = 0; oi < order.size() && rc == VR_OK; ++oi) {
        const std::vector<int>& members = buckets[order[oi].second];
        const int was = strategy_of(b->descs[members[0]]);
        for (int s = 0; s < kStrategies && rc == VR_OK; ++s) {
            if (s == was) continue;
            std::vector<BatchDesc> saved;
            bool ok = true;
            for (int i : members) {
                saved.push_back(b->descs[i]);
                ok = ok && apply_strategy(b, b->inst[i], b->descs[i], s);
            }
            double t = 0;
            if (ok && upload()) rc = measure(&t);
            if (!(ok && rc == VR_OK && t < cur * 0.995)) {  // keep a strategy only when it is faster
                for (size_t j = 0; j < members.size(); ++j) b->descs[members[j]] = saved[j];
            } else {
                cur = t;
            }
        }
        if (!upload()) rc = VR_ERR_CUDA;
    }
    // the chosen strategies: in the launch's counts, and in the autotuner's
    // table for each instance's (spec, rows, estimated groups) bucket
    b->info.whole_tables = b->info.caches = b->info.hbm_only = 0;
    for (int i = 0; i < n && rc == VR_OK; ++i) {
        const int s = strategy_of(b->descs[i]);
        (s == kWhole ? b->info.whole_tables : s == kHbm ? b->info.hbm_only : b->info.caches)++;
        vr_tune_choice c;
        std::memset(&c, 0, sizeof(c));
        c.tier = s == kHbm ? 2 : 1;
        c.warp_agg = b->descs[i].warp_agg;
        c.threads = b->cfg.consumer_threads;
        c.tile_rows = b->cfg.tile_rows;
        c.smem_slots = s == kWhole ? 0 : b->descs[i].smem_slots;  // 0: the default, a table of every group
        vr_tune_record(&b->inst[i]->spec, b->descs[i].num_rows, &c, (double)b->total_rows / (cur * 1e-3));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (best_ms) *best_ms = cur;
    return rc;
}

void vr_batched_destroy(vr_batched* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->descs_dev);
    cudaFree(b->spans_dev);
    cudaFree(b->counter);
    cudaFree(b->ctrl_all_dev);
    cudaFreeHost(b->ctrl_all_host);
    delete b;
}

}  // extern "C"
