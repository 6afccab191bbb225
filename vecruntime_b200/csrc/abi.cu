// C ABI of libvrgpu: handle lifecycle, staging, launches, growth, emission.
//
// The handle mirrors the reference's per-task aggregate state
// (VectorGroupedAggregateIterator, VectorHashAggregateExec.scala:463-1039):
// update = consume(batch) (:584-602), num_groups = table.size(), emit =
// buildBatch(from, to) (:831-913), reset = EmitAndReset (:193-246), destroy =
// close (:999-1019). One handle per task thread; each owns a CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "runtime.h"
#include "jit.h"
#include "tune.h"

namespace vr {

static thread_local std::string t_last_error;
void set_thread_error(const std::string& msg) { t_last_error = msg; }

int set_err(vr_agg* h, int code, const std::string& msg) {
    if (h) {
        if (h->status == VR_OK) {
            h->status = code;
            h->last_error = msg;
        }
        if (code != VR_ERR_INVALID && code != VR_ERR_UNSUPPORTED) h->dead = true;
    }
    t_last_error = msg;
    return code;
}

int cuda_err(vr_agg* h, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return VR_OK;
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return set_err(h, VR_ERR_OOM, msg);
    return set_err(h, VR_ERR_CUDA, msg);
}

static std::mutex g_dev_mu;
static DeviceInfo g_dev[64];

DeviceInfo& device_info(int device) {
    std::lock_guard<std::mutex> lk(g_dev_mu);
    DeviceInfo& d = g_dev[device & 63];
    if (!d.ready) {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device);
        cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
        cudaDeviceGetAttribute(&d.smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
        cudaDeviceGetAttribute(&d.smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock, device);
        cudaSetDevice(prev);
        d.ready = true;
    }
    return d;
}

int64_t next_pow2(int64_t x) {
    int64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}
static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int32_t stage_bytes_for(const Program& P, int T) {
    int32_t b = 0;
    for (int c = 0; c < P.num_cols; ++c) {
        int w = P.col_width[c];
        b += (int32_t)al256(w ? (size_t)T * w : (size_t)T / 8);
        if (P.col_nullable[c]) b += (int32_t)al256((size_t)T / 8);
    }
    b += (int32_t)al256((size_t)T / 8);  // selection
    return b;
}

void fill_layout(const Program& P, int T, StageLayout& L) {
    int32_t off = 0;
    for (int c = 0; c < kMaxCols; ++c) {
        L.data_off[c] = -1;
        L.valid_off[c] = -1;
    }
    for (int c = 0; c < P.num_cols; ++c) {
        int w = P.col_width[c];
        L.data_off[c] = off;
        off += (int32_t)al256(w ? (size_t)T * w : (size_t)T / 8);
        if (P.col_nullable[c]) {
            L.valid_off[c] = off;
            off += (int32_t)al256((size_t)T / 8);
        }
    }
    L.sel_off = off;
    off += (int32_t)al256((size_t)T / 8);
    L.stage_bytes = off;
}

int64_t tiles_for(const vr_agg* h, int64_t rows) { return (rows + h->cfg.tile_rows - 1) / h->cfg.tile_rows; }

// The aggregate launch: the spec's own kernel when it was compiled, else the
// interpreted ahead-of-time one.
cudaError_t agg_launch(vr_agg* h, const BatchDesc* descs, const LaunchCfg& L, int blocks, uint64_t* tile_counter,
                       cudaStream_t st) {
    if (h->jit) return jit_launch(h->jit, descs, L, blocks, tile_counter, st);
    return launch_aggregate(h->plan.prog.kw, h->cfg.tier, descs, L, blocks, tile_counter, st);
}

// CTAs per SM by default, and the most a choice may ask for.
constexpr int kDefaultCtasPerSm = 2;
constexpr int kMaxCtasPerSm = 4;

// How many CTAs of `threads` consumer threads (plus the producer warp), each
// with `smem` dynamic shared bytes and `regs` registers per thread (0 =
// unknown), fit on one SM together, at most `want`.
int ctas_per_sm(const DeviceInfo& di, int smem, int regs, int threads, int want) {
    const int block = threads + 32;
    const int rb = (regs + 7) / 8 * 8;
    int k = 1;
    while (k < want && di.fits(k + 1, smem) && (k + 1) * block <= 2048 && (regs <= 0 || (k + 1) * rb * block <= 65536))
        ++k;
    return k;
}

static int wanted_ctas(const vr_tune_choice* forced) {
    return forced && forced->blocks_per_sm ? std::min<int>(forced->blocks_per_sm, kMaxCtasPerSm) : kDefaultCtasPerSm;
}

// Picks tier, block shape, tile and shared-cache sizes. `forced` (tests /
// tuner) overrides the defaults field by field.
static int choose_config(vr_agg* h, const vr_tune_choice* forced) {
    const Program& P = h->plan.prog;
    const DeviceInfo& di = device_info(h->device);
    const int budget = di.smem_optin;
    const int fl = h->spec.flags;
    Config c;
    int64_t est = h->spec.est_groups > 0 ? h->spec.est_groups : 0;
    int want_tier = -1;  // from force flags / choice
    if (fl & VR_SPEC_FORCE_DIRECT) want_tier = 0;
    if (fl & VR_SPEC_FORCE_SHARED) want_tier = 1;
    if (fl & VR_SPEC_FORCE_GLOBAL) want_tier = 2;
    if (forced) want_tier = forced->tier;
    if (want_tier == 0 && !h->plan.direct_ok)
        return set_err(h, VR_ERR_UNSUPPORTED, "direct tier needs dictionary or boolean keys");

    auto fits = [&](int stages, int T, int tier_bytes) {
        return smem_map(stages, stage_bytes_for(P, T), tier_bytes).total <= budget;
    };
    bool chosen = false;
    if (h->plan.direct_ok && (want_tier == -1 || want_tier == 0)) {
        // A tile is exactly one chunk: threads x R rows (R rows per consumer
        // thread), so no lane idles inside a full tile. Among the shapes that
        // fit, the most consumer threads per SM times rows in flight per
        // thread (up to 4) wins, two CTAs per SM on a tie. Measured on the
        // decimal report (20M rows): 2 CTAs x 160 threads x 4 rows 0.297 ms,
        // 3 x 96 x 4 0.301 ms, 4 x 64 x 4 0.310 ms, 2 x 128 x 4 0.321 ms,
        // 1 x 256 x 4 0.35 ms, 1 x 224 x 4 0.37 ms, 2 x 96 x 4 0.38 ms,
        // 1 x 128 x 8 0.50 ms, 1 x 256 x 2 0.51 ms. More than two CTAs per SM
        // only on request (a tuning choice).
        const int nts[] = {256, 224, 192, 160, 128, 96, 64};
        const int Rs[] = {4, 8, 2};
        int64_t best = -1;
        const int top = wanted_ctas(forced);
        for (int ctas = top; ctas >= (forced && forced->blocks_per_sm ? top : 1); --ctas) {
            const int bytes = ctas == 1 ? budget : std::min(budget, di.smem_per_sm / ctas - di.smem_reserved);
            for (int nt : nts) {
                if (forced && forced->threads && nt != forced->threads) continue;
                // thread-private hot words + the CTA's cold words, for every
                // group and the trash group that rows which do not count go to
                int64_t tb = ((P.direct_slots + 1) * P.hw * (int64_t)nt + (P.direct_slots + 1) * P.aw) * 8;
                if (tb > bytes) continue;
                for (int R : Rs) {
                    const int T = nt * R;
                    if (T % 128) continue;
                    if (forced && forced->tile_rows && T != forced->tile_rows) continue;
                    for (int st = 3; st >= 2; --st) {
                        if (smem_map(st, stage_bytes_for(P, T), (int)tb).total > bytes) continue;
                        const int64_t score = (int64_t)ctas * nt * std::min(R, 4);
                        if (score > best) {  // strict: the first (two CTAs, more stages) keeps a tie
                            best = score;
                            c.tier = kTierDirect;
                            c.threads = nt;
                            c.tile_rows = T;
                            c.rchunk = R;
                            c.stages = st;
                            chosen = true;
                        }
                        break;
                    }
                }
            }
        }
        if (!chosen && want_tier == 0) return set_err(h, VR_ERR_UNSUPPORTED, "direct tier does not fit in shared memory");
    }
    if (!chosen) {
        c.tier = kTierHash;
        c.threads = forced && forced->threads ? forced->threads : 256;
        int64_t g = est > 0 ? est : std::min<int64_t>(h->spec.max_batch_rows > 0 ? h->spec.max_batch_rows : (1 << 20), 1 << 20);
        c.capacity = forced && forced->table_capacity ? next_pow2(forced->table_capacity) : next_pow2(std::max<int64_t>(1024, 2 * g));
        // one row per thread per step: unrolling the probe loops over several
        // rows overflows the instruction cache (measured 1.2x to 3.6x slower)
        c.rchunk = 1;
        const bool use_cache = want_tier != 2;
        const int64_t need = next_pow2(std::max<int64_t>(64, 2 * (est > 0 ? est : int64_t(1) << 30)));
        const int slot_bytes = 8 * P.sw;
        auto pow2_floor = [](int64_t x) {
            int64_t p = 1;
            while (p * 2 <= x) p *= 2;
            return x >= 1 ? p : 0;
        };
        // (tile rows, stages, shared slots) that fit in `bytes` of shared memory
        auto fit = [&](int T, int st, int bytes) -> int64_t {
            int used = smem_map(st, stage_bytes_for(P, T), 0).total;
            return used > bytes ? -1 : pow2_floor((bytes - used) / slot_bytes);
        };
        const int Ts[] = {2048, 1024, 512, 256};
        bool done = false;
        // 1) every group in a private per-CTA table, the longest tiles that leave
        //    room for it; two CTAs per SM when both fit (measured: a table that
        //    holds all groups is 2x faster than a cache that holds half of them)
        if (use_cache && !(forced && forced->smem_slots)) {
            const int half = di.smem_per_sm / 2 - di.smem_reserved;
            const bool wide = !(forced && forced->threads) && jit_enabled() && !(fl & VR_SPEC_NO_JIT) &&
                              !h->prebuilt_only;
            for (int ctas = 2; ctas >= 1 && !done; --ctas) {
                const int bytes = ctas == 2 ? std::min(half, budget) : budget;
                for (int T : Ts) {
                    if (forced && forced->tile_rows && T != forced->tile_rows) continue;
                    if (ctas == 1 && wide && T > 1024 && !(forced && forced->tile_rows)) continue;
                    for (int st = 3; st >= 2 && !done; --st) {
                        if (fit(T, st, bytes) >= need) {
                            c.tile_rows = T;
                            c.stages = st;
                            c.smem_slots = (int)need;
                            c.s_probes = 64;  // at most half full: every key finds its place
                            // one CTA per SM holds the whole table: give it 512
                            // consumer threads and 1,024-row tiles (measured on
                            // 40M rows into 1,000 groups: 1.31 ms, where 992
                            // threads take 1.43 and 768 with 768-row tiles 2.23;
                            // on 4M rows 512 threads took 0.20 ms, 256 0.34)
                            if (ctas == 1 && wide) c.threads = kWholeTableThreads;
                            done = true;
                        }
                    }
                    if (done) break;
                }
            }
        }
        // 2) otherwise two CTAs per SM with a hot-key cache in front of HBM
        //    (the first keys a CTA meets hold it; under skew those are the
        //    frequent ones). A bigger cache catches more of them but every
        //    CTA flushes all of it into HBM at the end, a fixed cost per
        //    launch (measured: 1,024 slots cost 33 us more than 256 on
        //    uniform keys), so the cache grows with the batch: 256 slots
        //    below 8M rows, 512 below 16M, then as many as two CTAs per SM
        //    leave room for; the tile is the longest that still fits it.
        //    Measured on Zipf(1.1) composite keys, 80-byte slots: 256-row
        //    tiles with 1,024 slots 2.45 ms per 20M rows (12.9 per 100M),
        //    512 x 512 2.64, 1024 x 256 2.86 (15.1), no cache 4.07.
        if (!done) {
            const int half = std::min(budget, di.smem_per_sm / 2 - di.smem_reserved);
            const int64_t rows = h->spec.max_batch_rows > 0 ? h->spec.max_batch_rows : (int64_t)1 << 20;
            int64_t want = 256;
            while (want < 4096 && want * 2 * 16384 <= rows) want *= 2;
            want = std::min<int64_t>(want, need);
            if (forced && forced->tile_rows) {
                c.tile_rows = forced->tile_rows;
            } else {
                c.tile_rows = 1024;
                while (c.tile_rows > 256 && fit(c.tile_rows, 3, half) < want) c.tile_rows /= 2;
            }
            c.stages = 3;
            while (c.stages > 2 && !fits(c.stages, c.tile_rows, 0)) --c.stages;
            while (!fits(c.stages, c.tile_rows, 0) && c.tile_rows > 256) c.tile_rows /= 2;
            const int64_t slots = fit(c.tile_rows, c.stages, budget);
            const int64_t slots2 = fit(c.tile_rows, c.stages, half);
            c.smem_slots = 0;
            if (use_cache && slots >= 64) {
                int64_t take = forced && forced->smem_slots ? next_pow2(forced->smem_slots)
                                                            : std::min<int64_t>(want, std::max<int64_t>(slots2, 64));
                c.smem_slots = (int)std::min(slots, take);
                // keys settle within two slots of home or not at all, so a miss
                // (most rows once the cache is full) costs two probes
                c.s_probes = 2;
            }
        }
        // warp pre-aggregation pays only when rows of a warp often share a
        // key: a handful of groups (measured: it costs 40% at 1,000 uniform
        // groups and 12% at millions of Zipf groups)
        c.warp_agg = (est > 0 && est <= 64) ? 1 : 0;
    }
    if (fl & VR_SPEC_WARP_AGG) c.warp_agg = 1;
    if (fl & VR_SPEC_NO_WARP_AGG) c.warp_agg = 0;
    if (forced) c.warp_agg = forced->warp_agg;
    if (fl & VR_SPEC_NO_TMA) c.tma = 0;
    const int tier_bytes = c.tier == kTierDirect
                               ? (int)(((P.direct_slots + 1) * P.hw * (int64_t)c.threads + (P.direct_slots + 1) * P.aw) * 8)
                               : c.smem_slots * P.sw * 8;
    SmemMap m = smem_map(c.stages, stage_bytes_for(P, c.tile_rows), tier_bytes);
    // blocks per SM: shared memory and registers (the ahead-of-time kernel's;
    // refined once a per-spec kernel is loaded)
    c.blocks_per_sm = ctas_per_sm(di, m.total, aggregate_kernel_regs(P.kw, c.tier), c.threads, wanted_ctas(forced));
    if (m.total > budget) return set_err(h, VR_ERR_UNSUPPORTED, "configuration exceeds shared memory");
    const bool jit_on = jit_enabled() && !(fl & VR_SPEC_NO_JIT) && !h->prebuilt_only;
    if (c.threads % 32 || c.threads > (jit_on ? kMaxConsumerThreadsJit : kMaxConsumerThreads) || c.tile_rows % 128)
        return set_err(h, VR_ERR_INVALID, "bad forced block shape");
    h->cfg = c;
    LaunchCfg& L = h->launch;
    std::memset(&L, 0, sizeof(L));
    L.tile_rows = c.tile_rows;
    L.rchunk = c.rchunk;
    // ~2 s at most per barrier wait (a stage normally arrives in microseconds);
    // the test hooks shorten it and stop the producer, so a test can watch a
    // wait run out and the error come back with the context still usable
    L.wait_polls = 2048;
    if (const char* e = std::getenv("VRGPU_TEST_WAIT_POLLS")) L.wait_polls = std::max(1, std::atoi(e));
    if (const char* e = std::getenv("VRGPU_TEST_STALL_PRODUCER")) L.test_stall = std::atoi(e) != 0;
    L.stages = c.stages;
    L.consumer_threads = c.threads;
    L.num_desc = 1;
    L.g_probes = c.g_probes;
    L.s_probes = c.s_probes;
    fill_layout(P, c.tile_rows, L.lay);
    L.tier_bytes = tier_bytes;
    L.smem_bytes = m.total;
    h->blocks = di.sms * c.blocks_per_sm;
    return VR_OK;
}

static int alloc_table(vr_agg* h) {
    const Program& P = h->plan.prog;
    int64_t slots = h->cfg.tier == kTierDirect ? P.direct_slots : h->cfg.capacity + 1;  // +1: sentinel side slot
    size_t bytes = (size_t)slots * P.sw * 8;
    cudaError_t e = cudaMalloc(&h->table, bytes);
    if (e != cudaSuccess) return cuda_err(h, e, "table allocation");
    e = cudaMemsetAsync(h->table, 0, bytes, h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "table clear");
    h->table_slots = slots;
    h->stats.table_capacity = h->cfg.tier == kTierDirect ? P.direct_slots : h->cfg.capacity;
    return VR_OK;
}

static int alloc_slot(vr_agg* h, StageSlot& s) {
    cudaError_t e;
    if ((e = cudaMallocHost(&s.desc_host, sizeof(BatchDesc))) != cudaSuccess) return cuda_err(h, e, "pinned desc");
    if ((e = cudaMalloc(&s.desc_dev, sizeof(BatchDesc))) != cudaSuccess) return cuda_err(h, e, "desc");
    if ((e = cudaMalloc(&s.ctrl_dev, CTRL_WORDS * 8)) != cudaSuccess) return cuda_err(h, e, "ctrl");
    if ((e = cudaMallocHost(&s.ctrl_host, CTRL_WORDS * 8)) != cudaSuccess) return cuda_err(h, e, "pinned ctrl");
    std::memset(s.ctrl_host, 0, CTRL_WORDS * 8);
    if ((e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming)) != cudaSuccess) return cuda_err(h, e, "event");
    if ((e = cudaEventCreate(&s.t0)) != cudaSuccess) return cuda_err(h, e, "event");
    if ((e = cudaEventCreate(&s.t1)) != cudaSuccess) return cuda_err(h, e, "event");
    if ((e = cudaEventCreate(&s.h0)) != cudaSuccess) return cuda_err(h, e, "event");
    if ((e = cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming)) != cudaSuccess) return cuda_err(h, e, "event");
    if (h->cfg.tier != kTierDirect) {
        // spill list: every shared slot of every CTA, the most one launch can spill
        s.spill_cap = (int64_t)h->blocks * std::max(1, h->cfg.smem_slots);
        if ((e = cudaMalloc(&s.spill, (size_t)s.spill_cap * h->plan.prog.sw * 8)) != cudaSuccess)
            return cuda_err(h, e, "spill list");
    }
    return VR_OK;
}

// Device staging for a host batch of n rows: every staged column and
// validity bitmap, plus the selection bitmap, each 256-byte aligned.
static size_t staging_bytes(const Program& P, int64_t n) {
    size_t need = 0;
    for (int c = 0; c < P.num_cols; ++c) {
        int w = P.col_width[c];
        need += al256(w ? (size_t)n * w : (size_t)(n + 7) / 8 + 4);
        need += al256((size_t)(n + 7) / 8 + 4);
    }
    return need + al256((size_t)(n + 7) / 8 + 4);
}

static int ensure_deferred(vr_agg* h, StageSlot& s, int64_t rows) {
    if (h->cfg.tier == kTierDirect || s.deferred_cap >= rows) return VR_OK;
    cudaFree(s.deferred);
    cudaFree(s.deferred_tmp);
    s.deferred = s.deferred_tmp = nullptr;
    int64_t cap = std::max<int64_t>(rows, 4096);
    cudaError_t e = cudaMalloc(&s.deferred, (size_t)cap * 8);
    if (e == cudaSuccess) e = cudaMalloc(&s.deferred_tmp, (size_t)cap * 8);
    if (e != cudaSuccess) return cuda_err(h, e, "deferred list");
    s.deferred_cap = cap;
    return VR_OK;
}

// Sizes both staging sets (host batches) and deferred-row lists for batches
// of up to `rows` rows now, so that no later update has to grow them: growing
// means cudaFree, which waits for the whole device, and a server issuing many
// queries' updates from one thread would stall on it.
int agg_reserve(vr_agg* h, int64_t rows) {
    if (rows <= 0) return VR_OK;
    cudaSetDevice(h->device);
    const size_t need = staging_bytes(h->plan.prog, rows);
    for (StageSlot& s : h->slot) {
        int rc = ensure_deferred(h, s, rows);
        if (rc != VR_OK) return rc;
        if (need <= s.dev_cap) continue;
        if (s.dev) {
            cudaError_t e = cudaFree(s.dev);
            if (e != cudaSuccess) return cuda_err(h, e, "staging free");
        }
        s.dev = nullptr;
        s.dev_cap = 0;
        cudaError_t e = cudaMalloc(&s.dev, need);
        if (e != cudaSuccess) return cuda_err(h, e, "staging allocation");
        s.dev_cap = need;
    }
    return VR_OK;
}

int agg_build(const vr_agg_spec* spec, const vr_tune_choice* forced, vr_agg** out, cudaStream_t stream) {
    if (!spec || !out) {
        set_thread_error("null argument");
        return VR_ERR_INVALID;
    }
    *out = nullptr;
    vr_agg* h = new (std::nothrow) vr_agg();
    if (!h) return VR_ERR_OOM;
    h->columns.assign(spec->columns, spec->columns + spec->num_columns);
    h->keys.assign(spec->key_columns, spec->key_columns + spec->num_keys);
    h->fns.assign(spec->fns, spec->fns + spec->num_fns);
    h->spec = *spec;
    h->spec.columns = h->columns.data();
    h->spec.key_columns = h->keys.data();
    h->spec.fns = h->fns.data();
    h->device = spec->device;
    h->trace = (spec->flags & VR_SPEC_TRACE) != 0;
    int rc = compile_plan(h->spec, h->plan);
    if (rc != VR_OK) {
        set_thread_error(h->plan.reason);
        delete h;
        return rc;
    }
    for (int k = 0; k < h->plan.prog.num_keys; ++k) {
        if (!h->plan.prog.keys[k].remap) continue;
        TableDict td;
        td.key = k;
        td.limit = h->columns[h->keys[k]].dict_size;
        h->tdicts.push_back(std::move(td));
    }
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) {
        set_thread_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        delete h;
        return VR_ERR_CUDA;
    }
    vr_tune_choice tuned;
    if (!forced && tune_lookup_internal(h->spec, h->spec.max_batch_rows, &tuned)) forced = &tuned;
    rc = choose_config(h, forced);
    if (rc != VR_OK) {
        std::string why = h->last_error;
        delete h;
        set_thread_error(why);
        return rc;
    }
    if (stream) {
        h->stream = stream;
    } else if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        set_thread_error(std::string("stream: ") + cudaGetErrorString(e));
        delete h;
        return VR_ERR_CUDA;
    } else {
        h->own_stream = true;
    }
    if ((e = cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) {
        set_thread_error(std::string("copy stream: ") + cudaGetErrorString(e));
        if (h->own_stream) cudaStreamDestroy(h->stream);
        delete h;
        return VR_ERR_CUDA;
    }
    h->stats.tier = h->cfg.tier == kTierDirect ? 0 : (h->cfg.smem_slots > 0 ? 1 : 2);
    h->stats.warp_agg = h->cfg.warp_agg;
    h->stats.slot_bytes = h->plan.prog.sw * 8;
    h->stats.threads = h->cfg.threads;
    h->stats.blocks = h->blocks;
    h->stats.smem_bytes = h->launch.smem_bytes;
    h->stats.tile_rows = h->cfg.tile_rows;
    // the spec's own kernel (compiled once per process per spec); the
    // interpreted ahead-of-time kernel stays the fallback
    if (jit_enabled() && !(spec->flags & VR_SPEC_NO_JIT)) {
        std::string why;
        const DeviceInfo& di = device_info(h->device);
        JitShape shape;
        shape.kw = h->plan.prog.kw;
        shape.tier = h->cfg.tier;
        shape.rchunk = h->cfg.rchunk;
        shape.threads = h->cfg.threads;
        // compiled for as many CTAs per SM as shared memory allows, up to the
        // wanted count (registers capped to fit)
        const int want = wanted_ctas(forced);
        shape.min_blocks = ctas_per_sm(di, h->launch.smem_bytes, 0, h->cfg.threads, want);
        shape.warp_agg = h->cfg.warp_agg;
        h->jit = jit_get(h->plan.prog, shape, h->device, &why);
        if (h->jit) {
            const int bps = ctas_per_sm(di, h->launch.smem_bytes, jit_regs(h->jit), h->cfg.threads, want);
            h->cfg.blocks_per_sm = bps;
            h->blocks = di.sms * bps;
            h->stats.blocks = h->blocks;
        } else {
            h->jit_error = why;
            if (h->cfg.threads > kMaxConsumerThreads) {
                // the prebuilt kernel's launch bounds cap the block: choose again for it
                h->prebuilt_only = true;
                if ((rc = choose_config(h, forced)) != VR_OK) {
                    std::string msg = h->last_error;
                    vr_agg_destroy(h);
                    set_thread_error(msg);
                    return rc;
                }
                h->stats.threads = h->cfg.threads;
                h->stats.blocks = h->blocks;
                h->stats.smem_bytes = h->launch.smem_bytes;
                h->stats.tile_rows = h->cfg.tile_rows;
            }
        }
    }
    h->stats.jit = h->jit ? 1 : 0;
    if ((e = cudaMalloc(&h->prog_dev, sizeof(Program))) != cudaSuccess ||
        (e = cudaMalloc(&h->emit_dev, sizeof(EmitProgram))) != cudaSuccess ||
        (e = cudaMemcpy(h->prog_dev, &h->plan.prog, sizeof(Program), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(h->emit_dev, &h->plan.emit, sizeof(EmitProgram), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&h->num_dev, 8)) != cudaSuccess ||
        (e = cudaMalloc(&h->outs_dev, sizeof(vr_out_column) * kMaxOut)) != cudaSuccess ||
        (e = cudaMallocHost(&h->outs_host, sizeof(vr_out_column) * kMaxOut)) != cudaSuccess ||
        (e = cudaMallocHost(&h->emit_ctrl, 64)) != cudaSuccess ||
        (e = cudaMallocHost(&h->aux_desc_host, sizeof(BatchDesc))) != cudaSuccess ||
        (e = cudaMalloc(&h->aux_desc_dev, sizeof(BatchDesc))) != cudaSuccess ||
        (e = cudaMalloc(&h->aux_ctrl_dev, CTRL_WORDS * 8)) != cudaSuccess ||
        (e = cudaMallocHost(&h->aux_ctrl_host, CTRL_WORDS * 8)) != cudaSuccess) {
        cuda_err(h, e, "handle allocation");
        std::string why = h->last_error;
        vr_agg_destroy(h);
        set_thread_error(why);
        return e == cudaErrorMemoryAllocation ? VR_ERR_OOM : VR_ERR_CUDA;
    }
    rc = alloc_table(h);
    for (int i = 0; i < 2 && rc == VR_OK; ++i) rc = alloc_slot(h, h->slot[i]);
    if (rc == VR_OK) {
        e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = cuda_err(h, e, "create");
    }
    if (rc != VR_OK) {
        std::string why = h->last_error;
        vr_agg_destroy(h);
        set_thread_error(why);
        return rc;
    }
    *out = h;
    return VR_OK;
}

// Batch -> staged column pointers (host batches are copied into slot memory).
static int stage_batch(vr_agg* h, StageSlot& s, const vr_batch& b, const char** data, const uint32_t** valid,
                       const uint32_t** sel) {
    const Plan& plan = h->plan;
    const Program& P = plan.prog;
    const int64_t n = b.num_rows;
    if (b.location == VR_DEVICE) {
        for (int c = 0; c < P.num_cols; ++c) {
            const vr_column& col = b.columns[plan.spec_of_staged[c]];
            data[c] = (const char*)col.data;
            valid[c] = (const uint32_t*)col.validity;
            if (((uintptr_t)col.validity & 3) != 0)
                return set_err(h, VR_ERR_INVALID, "validity bitmaps must be 4-byte aligned");
            if (!data[c] && n > 0) return set_err(h, VR_ERR_INVALID, "null column data");
        }
        *sel = (const uint32_t*)b.selection;
        if (((uintptr_t)b.selection & 3) != 0) return set_err(h, VR_ERR_INVALID, "selection must be 4-byte aligned");
        s.staged_h2d = false;
        return VR_OK;
    }
    // host batch: one H2D copy per buffer into the slot's staging area
    const size_t need = staging_bytes(P, n);
    if (need > s.dev_cap) {
        if (s.dev) {
            cudaError_t e = cudaFree(s.dev);
            if (e != cudaSuccess) return cuda_err(h, e, "staging free");
        }
        s.dev = nullptr;
        size_t cap = std::max(need, s.dev_cap + s.dev_cap / 2);
        cudaError_t e = cudaMalloc(&s.dev, cap);
        if (e != cudaSuccess) {
            s.dev_cap = 0;
            return cuda_err(h, e, "staging allocation");
        }
        s.dev_cap = cap;
    }
    cudaStream_t cs = h->copy_stream;
    // copies of this slot wait until the kernel that last read it is done
    if (s.pending_done_recorded) cudaStreamWaitEvent(cs, s.done, 0);
    if (h->trace) cudaEventRecord(s.h0, cs);
    size_t off = 0;
    int64_t bytes_in = 0;
    for (int c = 0; c < P.num_cols; ++c) {
        const vr_column& col = b.columns[plan.spec_of_staged[c]];
        int w = P.col_width[c];
        size_t db = w ? (size_t)n * w : (size_t)(n + 7) / 8;
        char* dst = s.dev + off;
        if (n > 0) {
            if (!col.data) return set_err(h, VR_ERR_INVALID, "null column data");
            cudaError_t e = cudaMemcpyAsync(dst, col.data, db, cudaMemcpyHostToDevice, cs);
            if (e != cudaSuccess) return cuda_err(h, e, "H2D");
            bytes_in += (int64_t)db;
        }
        data[c] = dst;
        off += al256(w ? (size_t)n * w : (size_t)(n + 7) / 8 + 4);
        if (col.validity && n > 0) {
            size_t vb = (size_t)(n + 7) / 8;
            cudaError_t e = cudaMemcpyAsync(s.dev + off, col.validity, vb, cudaMemcpyHostToDevice, cs);
            if (e != cudaSuccess) return cuda_err(h, e, "H2D");
            valid[c] = (const uint32_t*)(s.dev + off);
            bytes_in += (int64_t)vb;
        } else {
            valid[c] = nullptr;
        }
        off += al256((size_t)(n + 7) / 8 + 4);
    }
    if (b.selection && n > 0) {
        size_t vb = (size_t)(n + 7) / 8;
        cudaError_t e = cudaMemcpyAsync(s.dev + off, b.selection, vb, cudaMemcpyHostToDevice, cs);
        if (e != cudaSuccess) return cuda_err(h, e, "H2D");
        *sel = (const uint32_t*)(s.dev + off);
        bytes_in += (int64_t)vb;
    } else {
        *sel = nullptr;
    }
    // the kernel (on the compute stream) starts once this slot's copies landed;
    // the other slot's copies may meanwhile overlap the previous kernel
    cudaError_t e = cudaEventRecord(s.copied, cs);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->stream, s.copied, 0);
    if (e != cudaSuccess) return cuda_err(h, e, "copy ordering");
    s.staged_h2d = true;
    return VR_OK;
}

void fill_desc(vr_agg* h, const vr_batch& b, BatchDesc& d, uint64_t* ctrl, const StageSlot& s, int64_t tile_begin) {
    (void)b;
    d.num_rows = b.num_rows;
    d.tile_begin = tile_begin;
    d.num_tiles = tiles_for(h, b.num_rows);
    d.table = h->table;
    d.cap_mask = h->cfg.tier == kTierDirect ? h->plan.prog.direct_slots : h->cfg.capacity - 1;
    d.ctrl = ctrl;
    d.deferred = s.deferred;
    d.deferred_cap = s.deferred_cap;
    d.spill = s.spill;
    d.spill_cap = s.spill_cap;
    d.prog = h->prog_dev;
    d.tier = h->cfg.tier;
    d.smem_slots = h->cfg.smem_slots;
    d.warp_agg = h->cfg.warp_agg;
    d.s_probes = h->cfg.s_probes;
}

static bool tma_ok(const vr_agg* h, const BatchDesc& d) {
    if (!h->cfg.tma) return false;
    for (int c = 0; c < h->plan.prog.num_cols; ++c) {
        if (((uintptr_t)d.col_data[c] & 15) != 0) return false;
        if (d.col_valid[c] && ((uintptr_t)d.col_valid[c] & 15) != 0) return false;
    }
    if (d.selection && ((uintptr_t)d.selection & 15) != 0) return false;
    return true;
}

// Grows the HBM table to at least `need_groups` at load <= 1/2 and moves every
// group over (k_merge_slots). Stream-ordered; the caller synchronises.
static int grow_table(vr_agg* h, int64_t need_groups) {
    const Program& P = h->plan.prog;
    int64_t new_cap = std::max<int64_t>(2 * h->cfg.capacity, next_pow2(2 * need_groups));
    uint64_t* old = h->table;
    int64_t old_slots = h->table_slots;
    size_t bytes = (size_t)(new_cap + 1) * P.sw * 8;
    uint64_t* nt = nullptr;
    cudaError_t e = cudaMalloc(&nt, bytes);
    if (e != cudaSuccess) return cuda_err(h, e, "table grow");
    if ((e = cudaMemsetAsync(nt, 0, bytes, h->stream)) != cudaSuccess) return cuda_err(h, e, "table grow");
    h->table = nt;
    h->cfg.capacity = new_cap;
    h->table_slots = new_cap + 1;
    BatchDesc d;
    std::memset(&d, 0, sizeof(d));
    vr_batch dummy{};
    fill_desc(h, dummy, d, h->aux_ctrl_dev, h->slot[0], 0);
    *h->aux_desc_host = d;
    if ((e = cudaMemcpyAsync(h->aux_desc_dev, h->aux_desc_host, sizeof(BatchDesc), cudaMemcpyHostToDevice, h->stream)) !=
        cudaSuccess)
        return cuda_err(h, e, "desc");
    if ((e = cudaMemsetAsync(h->aux_ctrl_dev, 0, CTRL_WORDS * 8, h->stream)) != cudaSuccess) return cuda_err(h, e, "ctrl");
    if ((e = launch_merge_slots(P.kw, h->aux_desc_dev, old, old_slots, (int)std::min<int64_t>(new_cap, 1 << 20),
                                h->stream)) != cudaSuccess)
        return cuda_err(h, e, "rehash");
    h->stats.kernel_launches++;
    if ((e = cudaMemcpyAsync(h->aux_ctrl_host, h->aux_ctrl_dev, CTRL_WORDS * 8, cudaMemcpyDeviceToHost, h->stream)) !=
        cudaSuccess)
        return cuda_err(h, e, "ctrl");
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "rehash");
    if (h->aux_ctrl_host[CTRL_ERROR]) return set_err(h, VR_ERR_OOM, "rehash could not place every group");
    cudaFree(old);
    h->groups_known = (int64_t)h->aux_ctrl_host[CTRL_GROUPS];
    h->stats.table_capacity = new_cap;
    h->stats.rehashes++;
    return VR_OK;
}

static int map_ctrl_error(vr_agg* h, uint64_t bits) {
    if (bits & kErrBadKey) return set_err(h, VR_ERR_INVALID, "dictionary id outside its declared dictionary size");
    if (bits & (kErrTimeout | kErrLockTimeout)) return set_err(h, VR_ERR_TIMEOUT, "a bounded device wait gave up");
    if (bits & (kErrDeferredFull | kErrSpillFull)) return set_err(h, VR_ERR_OOM, "deferred/spill list overflow");
    return set_err(h, VR_ERR_CUDA, "device error");
}

// Resolves every launched batch: errors, group counts, and rows or slots the
// HBM table could not take (grow, merge spills, replay deferred rows).
int agg_resolve_all(vr_agg* h) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "update");
    h->clear_queued = false;
    const Program& P = h->plan.prog;
    int order[2] = {h->next_slot, h->next_slot ^ 1};  // oldest first
    for (int k = 0; k < 2; ++k) {
        StageSlot& s = h->slot[order[k]];
        if (!s.pending) continue;
        s.pending = false;
        if (s.ctrl_host[CTRL_ERROR]) return map_ctrl_error(h, s.ctrl_host[CTRL_ERROR]);
        h->groups_known += (int64_t)s.ctrl_host[CTRL_GROUPS];
        if (s.timed) {
            float ms = 0;
            cudaEventElapsedTime(&ms, s.t0, s.t1);
            h->stats.last_kernel_ms = ms;
            h->stats.total_kernel_ms += ms;
            if (s.staged_h2d) {
                float hm = 0;
                cudaEventElapsedTime(&hm, s.h0, s.t0);
                h->stats.total_h2d_ms += hm;
            }
            s.timed = false;
        }
        int64_t deferred = (int64_t)s.ctrl_host[CTRL_DEFERRED];
        int64_t spilled = (int64_t)s.ctrl_host[CTRL_SPILLED];
        int guard = 0;
        while ((deferred > 0 || spilled > 0) && guard++ < 8) {
            int rc = grow_table(h, h->groups_known + deferred + spilled);
            if (rc != VR_OK) return rc;
            // the slot's batch descriptor, repointed at the grown table
            BatchDesc d = s.launched;
            d.table = h->table;
            d.cap_mask = h->cfg.capacity - 1;
            *s.desc_host = d;
            if ((e = cudaMemcpyAsync(s.desc_dev, s.desc_host, sizeof(BatchDesc), cudaMemcpyHostToDevice, h->stream)) !=
                cudaSuccess)
                return cuda_err(h, e, "desc");
            if (spilled > 0) {
                if ((e = cudaMemsetAsync(s.ctrl_dev, 0, CTRL_WORDS * 8, h->stream)) != cudaSuccess)
                    return cuda_err(h, e, "ctrl");
                if ((e = launch_merge_slots(P.kw, s.desc_dev, s.spill, std::min(spilled, s.spill_cap), h->cfg.g_probes,
                                            h->stream)) != cudaSuccess)
                    return cuda_err(h, e, "spill merge");
                h->stats.kernel_launches++;
                if ((e = cudaMemcpyAsync(s.ctrl_host, s.ctrl_dev, CTRL_WORDS * 8, cudaMemcpyDeviceToHost, h->stream)) !=
                    cudaSuccess)
                    return cuda_err(h, e, "ctrl");
                if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "spill merge");
                if (s.ctrl_host[CTRL_ERROR]) return map_ctrl_error(h, s.ctrl_host[CTRL_ERROR]);
                h->groups_known += (int64_t)s.ctrl_host[CTRL_GROUPS];
                spilled = 0;
            }
            if (deferred > 0) {
                int64_t n = std::min(deferred, s.deferred_cap);
                h->stats.deferred_rows += n;
                if ((e = cudaMemcpyAsync(s.deferred_tmp, s.deferred, (size_t)n * 8, cudaMemcpyDeviceToDevice,
                                         h->stream)) != cudaSuccess)
                    return cuda_err(h, e, "deferred copy");
                if ((e = cudaMemsetAsync(s.ctrl_dev, 0, CTRL_WORDS * 8, h->stream)) != cudaSuccess)
                    return cuda_err(h, e, "ctrl");
                if ((e = launch_replay(P.kw, s.desc_dev, s.deferred_tmp, n, h->cfg.g_probes, h->stream)) != cudaSuccess)
                    return cuda_err(h, e, "replay");
                h->stats.kernel_launches++;
                if ((e = cudaMemcpyAsync(s.ctrl_host, s.ctrl_dev, CTRL_WORDS * 8, cudaMemcpyDeviceToHost, h->stream)) !=
                    cudaSuccess)
                    return cuda_err(h, e, "ctrl");
                if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "replay");
                if (s.ctrl_host[CTRL_ERROR]) return map_ctrl_error(h, s.ctrl_host[CTRL_ERROR]);
                h->groups_known += (int64_t)s.ctrl_host[CTRL_GROUPS];
                deferred = (int64_t)s.ctrl_host[CTRL_DEFERRED];
            }
        }
        if (deferred > 0 || spilled > 0) return set_err(h, VR_ERR_OOM, "table growth did not converge");
    }
    return VR_OK;
}

// A column the spec declares non-nullable must not bring a validity bitmap:
// the kernels skip the validity test for such columns.
const char* batch_nullability_error(const vr_agg* h, const vr_batch& b) {
    for (int c = 0; c < h->plan.prog.num_cols; ++c) {
        const int sc = h->plan.spec_of_staged[c];
        if (!h->columns[sc].nullable && b.columns[sc].validity)
            return "a column declared non-nullable carries a validity bitmap";
    }
    return nullptr;
}

// Maps the batch dictionary of every VR_COL_BATCH_DICTIONARY key onto the
// key's table dictionary (one probe per dictionary entry, new strings get the
// next table id; GroupKeyTable.toIds, GroupKeyTable.java:1308-1430) and points
// the launch's descriptor at the maps, copied to the device on the handle's
// stream ahead of the kernel. Dictionaries of device batches are read back
// first (they are small next to the batch).
static int map_batch_dictionaries(vr_agg* h, StageSlot& s, const vr_batch& b, BatchDesc& d) {
    if (h->tdicts.empty()) return VR_OK;
    int64_t need = 0;
    for (const TableDict& td : h->tdicts) {
        const vr_column& col = b.columns[h->spec.key_columns[td.key]];
        if (!col.dictionary) return set_err(h, VR_ERR_INVALID, "a key declared with batch dictionaries came without one");
        if (col.dictionary->size < 0) return set_err(h, VR_ERR_INVALID, "negative dictionary size");
        need += col.dictionary->size;
    }
    cudaError_t e;
    if (need > s.remap_cap) {
        cudaFree(s.remap_dev);
        cudaFreeHost(s.remap_host);
        s.remap_dev = nullptr;
        s.remap_host = nullptr;
        s.remap_cap = 0;
        const int64_t cap = std::max<int64_t>(need, 1024);
        if ((e = cudaMalloc(&s.remap_dev, (size_t)cap * 4)) != cudaSuccess) return cuda_err(h, e, "dictionary maps");
        if ((e = cudaMallocHost(&s.remap_host, (size_t)cap * 4)) != cudaSuccess) return cuda_err(h, e, "dictionary maps");
        s.remap_cap = cap;
    }
    int64_t off = 0;
    std::vector<int32_t> offs;
    std::vector<uint8_t> bytes, valid;
    for (TableDict& td : h->tdicts) {
        const vr_dictionary& dict = *b.columns[h->spec.key_columns[td.key]].dictionary;
        const int32_t n = dict.size;
        const int32_t* o = dict.offsets;
        const uint8_t* data = dict.data;
        const uint8_t* vb = dict.validity;
        if (n > 0 && (!o || !data)) return set_err(h, VR_ERR_INVALID, "dictionary without offsets or data");
        if (n > 0 && b.location == VR_DEVICE) {  // read the device dictionary back
            offs.resize((size_t)n + 1);
            if ((e = cudaMemcpy(offs.data(), o, ((size_t)n + 1) * 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
                return cuda_err(h, e, "dictionary read-back");
            bytes.resize((size_t)std::max(0, offs[n] - offs[0]) + 1);
            if (offs[n] > offs[0] &&
                (e = cudaMemcpy(bytes.data(), data + offs[0], (size_t)(offs[n] - offs[0]), cudaMemcpyDeviceToHost)) !=
                    cudaSuccess)
                return cuda_err(h, e, "dictionary read-back");
            if (vb) {
                valid.resize((size_t)(n + 7) / 8);
                if ((e = cudaMemcpy(valid.data(), vb, valid.size(), cudaMemcpyDeviceToHost)) != cudaSuccess)
                    return cuda_err(h, e, "dictionary read-back");
                vb = valid.data();
            }
            for (int32_t k = n; k >= 0; --k) offs[k] -= offs[0];  // the bytes were read from offs[0] on
            data = bytes.data();
            o = offs.data();
        }
        int32_t* m = s.remap_host + off;
        for (int32_t k = 0; k < n; ++k) {
            if (vb && !((vb[k >> 3] >> (k & 7)) & 1)) {  // a null entry: its rows are null
                m[k] = -1;
                continue;
            }
            if (o[k + 1] < o[k]) return set_err(h, VR_ERR_INVALID, "dictionary offsets decrease");
            std::string str(reinterpret_cast<const char*>(data + o[k]), (size_t)(o[k + 1] - o[k]));
            auto it = td.ids.find(str);
            if (it == td.ids.end()) {
                const int32_t id = (int32_t)td.ids.size();
                if (td.limit > 0 && id >= td.limit)
                    return set_err(h, VR_ERR_INVALID, "more distinct strings than the key's declared dictionary size");
                it = td.ids.emplace(str, id).first;
                td.bytes += str;
                td.offsets.push_back((int32_t)td.bytes.size());
            }
            m[k] = it->second;
        }
        const int c = h->plan.prog.keys[td.key].col;
        d.col_remap[c] = s.remap_dev + off;
        d.col_remap_n[c] = n;
        off += n;
    }
    if (off > 0 && (e = cudaMemcpyAsync(s.remap_dev, s.remap_host, (size_t)off * 4, cudaMemcpyHostToDevice,
                                        h->stream)) != cudaSuccess)
        return cuda_err(h, e, "dictionary maps");
    return VR_OK;
}

static int agg_update(vr_agg* h, const vr_batch* b) {
    if (h->dead) return VR_ERR_STATE;
    if (!b || b->num_rows < 0 || (b->num_rows > 0 && !b->columns))
        return set_err(h, VR_ERR_INVALID, "bad batch");
    if (b->num_rows == 0) return VR_OK;
    if (const char* why = batch_nullability_error(h, *b)) return set_err(h, VR_ERR_INVALID, why);
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_err(h, e, "cudaSetDevice");
    StageSlot& s = h->slot[h->next_slot];
    if (s.pending) {  // the batch that used this staging set two updates ago
        if ((e = cudaEventSynchronize(s.done)) != cudaSuccess) return cuda_err(h, e, "update");
        bool needs = s.ctrl_host[CTRL_ERROR] || s.ctrl_host[CTRL_DEFERRED] || s.ctrl_host[CTRL_SPILLED];
        if (needs) {
            int rc = agg_resolve_all(h);
            if (rc != VR_OK) return rc;
        } else {
            s.pending = false;
            h->groups_known += (int64_t)s.ctrl_host[CTRL_GROUPS];
            if (s.timed) {
                float ms = 0;
                cudaEventElapsedTime(&ms, s.t0, s.t1);
                h->stats.last_kernel_ms = ms;
                h->stats.total_kernel_ms += ms;
                if (s.staged_h2d) {
                    float hm = 0;
                    cudaEventElapsedTime(&hm, s.h0, s.t0);
                    h->stats.total_h2d_ms += hm;
                }
                s.timed = false;
            }
        }
    }
    // keep the HBM table at load <= 1/2 of what is already known
    if (h->cfg.tier != kTierDirect && h->groups_known * 2 > h->cfg.capacity) {
        int rc = agg_resolve_all(h);
        if (rc == VR_OK) rc = grow_table(h, h->groups_known);
        if (rc != VR_OK) return rc;
    }
    int rc = ensure_deferred(h, s, b->num_rows);
    if (rc != VR_OK) return rc;
    BatchDesc d;
    std::memset(&d, 0, sizeof(d));
    const char* data[kMaxCols] = {};
    const uint32_t* valid[kMaxCols] = {};
    const uint32_t* sel = nullptr;
    rc = stage_batch(h, s, *b, data, valid, &sel);
    if (rc != VR_OK) return rc;
    for (int c = 0; c < kMaxCols; ++c) {
        d.col_data[c] = data[c];
        d.col_valid[c] = valid[c];
    }
    d.selection = sel;
    fill_desc(h, *b, d, s.ctrl_dev, s, 0);
    d.tma = tma_ok(h, d) ? 1 : 0;
    if ((rc = map_batch_dictionaries(h, s, *b, d)) != VR_OK) return rc;
    *s.desc_host = d;
    s.launched = d;
    if ((e = cudaMemcpyAsync(s.desc_dev, s.desc_host, sizeof(BatchDesc), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
        return cuda_err(h, e, "desc");
    if ((e = cudaMemsetAsync(s.ctrl_dev, 0, CTRL_WORDS * 8, h->stream)) != cudaSuccess) return cuda_err(h, e, "ctrl");
    LaunchCfg L = h->launch;
    L.total_tiles = d.num_tiles;
    int blocks = (int)std::min<int64_t>(h->blocks, d.num_tiles);
    if (h->trace) cudaEventRecord(s.t0, h->stream);
    if ((e = agg_launch(h, s.desc_dev, L, blocks, &s.ctrl_dev[CTRL_NEXT_TILE], h->stream)) != cudaSuccess)
        return cuda_err(h, e, "aggregate launch");
    if (h->trace) {
        cudaEventRecord(s.t1, h->stream);
        s.timed = true;
    }
    h->stats.kernel_launches++;
    if ((e = cudaMemcpyAsync(s.ctrl_host, s.ctrl_dev, CTRL_WORDS * 8, cudaMemcpyDeviceToHost, h->stream)) != cudaSuccess)
        return cuda_err(h, e, "ctrl");
    if ((e = cudaEventRecord(s.done, h->stream)) != cudaSuccess) return cuda_err(h, e, "event");
    s.pending_done_recorded = true;
    s.pending = true;
    s.rows = b->num_rows;
    h->next_slot ^= 1;
    h->compact_valid = false;
    h->stats.rows += b->num_rows;
    h->stats.batches++;
    return VR_OK;
}

static int agg_compact(vr_agg* h) {
    int rc = agg_resolve_all(h);
    if (rc != VR_OK) return rc;
    if (h->compact_valid) return VR_OK;
    const Program& P = h->plan.prog;
    cudaError_t e;
    if (h->slot_of_cap < h->table_slots) {
        cudaFree(h->slot_of);
        h->slot_of = nullptr;
        if ((e = cudaMalloc(&h->slot_of, (size_t)h->table_slots * 8)) != cudaSuccess) return cuda_err(h, e, "compaction");
        h->slot_of_cap = h->table_slots;
    }
    size_t need = 0;
    if ((e = launch_compact_kw(P.kw, h->table, h->table_slots, P.sw, h->slot_of, h->num_dev, nullptr, &need, h->stream)) !=
        cudaSuccess)
        return cuda_err(h, e, "compaction sizing");
    if (need > h->cub_temp_bytes) {
        cudaFree(h->cub_temp);
        h->cub_temp = nullptr;
        if ((e = cudaMalloc(&h->cub_temp, need)) != cudaSuccess) return cuda_err(h, e, "compaction scratch");
        h->cub_temp_bytes = need;
    }
    size_t tb = h->cub_temp_bytes;
    if ((e = launch_compact_kw(P.kw, h->table, h->table_slots, P.sw, h->slot_of, h->num_dev, h->cub_temp, &tb,
                               h->stream)) != cudaSuccess)
        return cuda_err(h, e, "compaction");
    h->stats.kernel_launches += 2;
    int64_t n = 0;
    if ((e = cudaMemcpyAsync(h->emit_ctrl, h->num_dev, 8, cudaMemcpyDeviceToHost, h->stream)) != cudaSuccess)
        return cuda_err(h, e, "compaction");
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "compaction");
    n = (int64_t)h->emit_ctrl[0];
    h->num_groups = n;
    h->stats.groups = n;
    h->compact_valid = true;
    return VR_OK;
}

static size_t out_data_bytes(int lane, int64_t n) {
    switch (lane) {
        case VR_INT32:
        case VR_DICT32: return (size_t)n * 4;
        case VR_INT64:
        case VR_FLOAT64: return (size_t)n * 8;
        case VR_DECIMAL128: return (size_t)n * 16;
        case VR_BOOL: return (size_t)(n + 7) / 8;
    }
    return 0;
}

static int agg_emit(vr_agg* h, int64_t from, int64_t to, const vr_out_column* outs, int32_t location) {
    if (h->dead) return VR_ERR_STATE;
    int rc = agg_compact(h);
    if (rc != VR_OK) return rc;
    if (from < 0 || to < from || to > h->num_groups) return set_err(h, VR_ERR_INVALID, "emit range outside [0, groups]");
    if (!outs) return set_err(h, VR_ERR_INVALID, "null output columns");
    const int64_t n = to - from;
    if (n == 0) return VR_OK;
    const EmitProgram& E = h->plan.emit;
    cudaError_t e;
    if (location == VR_DEVICE) {
        for (int j = 0; j < E.num_out; ++j) h->outs_host[j] = outs[j];
    } else {
        size_t need = 0;
        for (int j = 0; j < E.num_out; ++j)
            need += al256(out_data_bytes(E.outs[j].lane, n)) + al256((size_t)(n + 7) / 8);
        if (need > h->emit_stage_cap) {
            cudaFree(h->emit_stage);
            h->emit_stage = nullptr;
            if ((e = cudaMalloc(&h->emit_stage, need)) != cudaSuccess) return cuda_err(h, e, "emit staging");
            h->emit_stage_cap = need;
        }
        size_t off = 0;
        for (int j = 0; j < E.num_out; ++j) {
            h->outs_host[j].data = h->emit_stage + off;
            off += al256(out_data_bytes(E.outs[j].lane, n));
            h->outs_host[j].validity = (uint8_t*)(h->emit_stage + off);
            off += al256((size_t)(n + 7) / 8);
        }
    }
    if ((e = cudaMemcpyAsync(h->outs_dev, h->outs_host, sizeof(vr_out_column) * E.num_out, cudaMemcpyHostToDevice,
                             h->stream)) != cudaSuccess)
        return cuda_err(h, e, "emit");
    if ((e = cudaMemsetAsync(h->aux_ctrl_dev, 0, CTRL_WORDS * 8, h->stream)) != cudaSuccess) return cuda_err(h, e, "ctrl");
    if ((e = launch_emit(h->prog_dev, h->emit_dev, h->table, h->slot_of, from, to, h->outs_dev, h->aux_ctrl_dev,
                         h->stream)) !=
        cudaSuccess)
        return cuda_err(h, e, "emit launch");
    h->stats.kernel_launches++;
    if (location != VR_DEVICE) {
        for (int j = 0; j < E.num_out; ++j) {
            if (outs[j].data) {
                e = cudaMemcpyAsync(outs[j].data, h->outs_host[j].data, out_data_bytes(E.outs[j].lane, n),
                                    cudaMemcpyDeviceToHost, h->stream);
                if (e != cudaSuccess) return cuda_err(h, e, "D2H");
            }
            if (outs[j].validity) {
                e = cudaMemcpyAsync(outs[j].validity, h->outs_host[j].validity, (size_t)(n + 7) / 8,
                                    cudaMemcpyDeviceToHost, h->stream);
                if (e != cudaSuccess) return cuda_err(h, e, "D2H");
            }
        }
    }
    if ((e = cudaMemcpyAsync(h->aux_ctrl_host, h->aux_ctrl_dev, CTRL_WORDS * 8, cudaMemcpyDeviceToHost, h->stream)) !=
        cudaSuccess)
        return cuda_err(h, e, "ctrl");
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "emit");
    int st = (int)h->aux_ctrl_host[CTRL_EMIT_ERROR];
    if (st != 0) {
        const char* why = st == VR_ERR_OVERFLOW ? "long overflow (ANSI sum)"
                          : st == VR_ERR_DECIMAL_OVERFLOW ? "overflow in sum of decimals (ANSI)"
                                                          : "decimal result past its precision (ANSI)";
        return set_err(h, st, why);
    }
    return VR_OK;
}

}  // namespace vr

using namespace vr;

extern "C" {

int vr_agg_create(const vr_agg_spec* spec, vr_agg** out) { return agg_build(spec, nullptr, out, nullptr); }

int vr_agg_create_tuned(const vr_agg_spec* spec, const vr_tune_choice* choice, vr_agg** out) {
    return agg_build(spec, choice, out, nullptr);
}

int vr_agg_update(vr_agg* h, const vr_batch* b) {
    if (!h) return VR_ERR_INVALID;
    return agg_update(h, b);
}

int vr_agg_sync(vr_agg* h) {
    if (!h) return VR_ERR_INVALID;
    if (h->dead) return VR_ERR_STATE;
    cudaSetDevice(h->device);
    return agg_resolve_all(h);
}

int vr_agg_num_groups(vr_agg* h, int64_t* groups) {
    if (!h || !groups) return VR_ERR_INVALID;
    if (h->dead) return VR_ERR_STATE;
    cudaSetDevice(h->device);
    int rc = agg_compact(h);
    if (rc == VR_OK) *groups = h->num_groups;
    return rc;
}

int vr_agg_output_schema(const vr_agg* h, int32_t* num_out, vr_column_type* types, int32_t cap) {
    if (!h || !num_out) return VR_ERR_INVALID;
    *num_out = (int32_t)h->plan.out_types.size();
    if (types)
        for (int32_t i = 0; i < *num_out && i < cap; ++i) types[i] = h->plan.out_types[i];
    return VR_OK;
}

int vr_agg_emit(vr_agg* h, int64_t from, int64_t to, const vr_out_column* outs, int32_t location) {
    if (!h) return VR_ERR_INVALID;
    cudaSetDevice(h->device);
    return agg_emit(h, from, to, outs, location);
}

int vr_agg_reset(vr_agg* h) {
    if (!h) return VR_ERR_INVALID;
    if (h->dead) return VR_ERR_STATE;
    cudaSetDevice(h->device);
    // a pending batch may still grow the table or fail: settle it first;
    // otherwise the clear is only queued behind earlier work on the stream
    // (later updates and emits are ordered after it), so the device never
    // idles while the host prepares the next launch
    if (h->slot[0].pending || h->slot[1].pending) {
        int rc = agg_resolve_all(h);
        if (rc != VR_OK) return rc;
    }
    cudaError_t e = cudaMemsetAsync(h->table, 0, (size_t)h->table_slots * h->plan.prog.sw * 8, h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "reset");
    h->clear_queued = true;
    for (TableDict& td : h->tdicts) {  // the emptied table's ids start again from 0
        td.ids.clear();
        td.offsets.assign(1, 0);
        td.bytes.clear();
    }
    h->groups_known = 0;
    h->compact_valid = false;
    h->num_groups = 0;
    return VR_OK;
}

void vr_agg_destroy(vr_agg* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& s : h->slot) {
        cudaFree(s.dev);
        cudaFreeHost(s.desc_host);
        cudaFree(s.desc_dev);
        cudaFree(s.ctrl_dev);
        cudaFreeHost(s.ctrl_host);
        cudaFree(s.deferred);
        cudaFree(s.deferred_tmp);
        cudaFree(s.spill);
        cudaFree(s.remap_dev);
        cudaFreeHost(s.remap_host);
        if (s.done) cudaEventDestroy(s.done);
        if (s.t0) cudaEventDestroy(s.t0);
        if (s.t1) cudaEventDestroy(s.t1);
        if (s.h0) cudaEventDestroy(s.h0);
        if (s.copied) cudaEventDestroy(s.copied);
    }
    cudaFree(h->table);
    cudaFree(h->prog_dev);
    cudaFree(h->emit_dev);
    cudaFree(h->slot_of);
    cudaFree(h->num_dev);
    cudaFree(h->cub_temp);
    cudaFree(h->outs_dev);
    cudaFreeHost(h->outs_host);
    cudaFree(h->emit_stage);
    cudaFreeHost(h->emit_ctrl);
    cudaFreeHost(h->aux_desc_host);
    cudaFree(h->aux_desc_dev);
    cudaFree(h->aux_ctrl_dev);
    cudaFreeHost(h->aux_ctrl_host);
    if (h->copy_stream) {
        cudaStreamSynchronize(h->copy_stream);
        cudaStreamDestroy(h->copy_stream);
    }
    if (h->stream && h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
}

int vr_agg_get_stats(const vr_agg* h, vr_agg_stats* st) {
    if (!h || !st) return VR_ERR_INVALID;
    *st = h->stats;
    st->groups = h->compact_valid ? h->num_groups : h->groups_known;
    return VR_OK;
}

int vr_agg_last_error(const vr_agg* h, char* buf, size_t cap) {
    if (!h || !buf || cap == 0) return VR_ERR_INVALID;
    std::snprintf(buf, cap, "%s", h->last_error.c_str());
    return VR_OK;
}

const char* vr_thread_last_error(void) { return t_last_error.c_str(); }

int vr_agg_error_value(const vr_agg* h, int64_t* lo, int64_t* hi, int32_t* precision, int32_t* scale) {
    if (!h || !lo || !hi || !precision || !scale) return VR_ERR_INVALID;
    const uint64_t ty = h->aux_ctrl_host ? h->aux_ctrl_host[CTRL_EMIT_VALUE_TYPE] : 0;
    if (h->status != VR_ERR_DECIMAL_PRECISION || !(ty >> 63)) return VR_ERR_STATE;
    *lo = (int64_t)h->aux_ctrl_host[CTRL_EMIT_VALUE_LO];
    *hi = (int64_t)h->aux_ctrl_host[CTRL_EMIT_VALUE_HI];
    *precision = (int32_t)((ty >> 32) & 0x7fffffff);
    *scale = (int32_t)(uint32_t)ty;
    return VR_OK;
}

int vr_agg_key_dictionary(const vr_agg* h, int32_t key, int32_t* size, int32_t* offsets, uint8_t* data,
                          int64_t data_cap, int64_t* data_bytes) {
    if (!h || !size) return VR_ERR_INVALID;
    for (const TableDict& td : h->tdicts) {
        if (td.key != key) continue;
        *size = (int32_t)td.ids.size();
        if (data_bytes) *data_bytes = (int64_t)td.bytes.size();
        if (offsets) std::memcpy(offsets, td.offsets.data(), td.offsets.size() * 4);
        if (data) {
            if (data_cap < (int64_t)td.bytes.size()) {
                t_last_error = "vr_agg_key_dictionary: data buffer smaller than the dictionary's bytes";
                return VR_ERR_INVALID;
            }
            std::memcpy(data, td.bytes.data(), td.bytes.size());
        }
        return VR_OK;
    }
    t_last_error = "vr_agg_key_dictionary: the key does not bring batch dictionaries";
    return VR_ERR_INVALID;
}

const char* vr_status_string(int s) {
    switch (s) {
        case VR_OK: return "ok";
        case VR_ERR_INVALID: return "invalid argument";
        case VR_ERR_OOM: return "out of memory";
        case VR_ERR_OVERFLOW: return "arithmetic overflow";
        case VR_ERR_DECIMAL_PRECISION: return "decimal precision exceeded";
        case VR_ERR_TIMEOUT: return "device wait timed out";
        case VR_ERR_CUDA: return "CUDA error";
        case VR_ERR_UNSUPPORTED: return "unsupported on the GPU";
        case VR_ERR_STATE: return "handle is dead or call out of order";
        case VR_ERR_ADMISSION: return "request exceeds the admission cap";
        case VR_ERR_DECIMAL_OVERFLOW: return "overflow in sum of decimals";
    }
    return "unknown status";
}

void* vr_agg_stream(const vr_agg* h) { return h ? (void*)h->stream : nullptr; }

int vr_host_alloc(size_t bytes, void** out) {
    if (!out) return VR_ERR_INVALID;
    cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        t_last_error = cudaGetErrorString(e);
        return VR_ERR_OOM;
    }
    return VR_OK;
}
int vr_host_free(void* p) { return cudaFreeHost(p) == cudaSuccess ? VR_OK : VR_ERR_CUDA; }
int vr_host_register(void* p, size_t bytes) {
    cudaError_t e = cudaHostRegister(p, bytes, cudaHostRegisterPortable);
    if (e != cudaSuccess) {
        t_last_error = cudaGetErrorString(e);
        return VR_ERR_CUDA;
    }
    return VR_OK;
}
int vr_host_unregister(void* p) { return cudaHostUnregister(p) == cudaSuccess ? VR_OK : VR_ERR_CUDA; }

}  // extern "C"

namespace vr {
// The kernel's descriptor of key column c (hashes: the dictionary's entry
// hashes for a VR_DICT32 key); an error message when the column cannot be
// hashed as the reference hashes it.
static const char* hash_key_of(const vr_column_type& t, const vr_column& k, const uint32_t* hashes, HashKey& out) {
    std::memset(&out, 0, sizeof(out));
    out.data = k.data;
    out.validity = k.validity;
    out.lane = t.lane;
    switch (t.lane) {
        case VR_INT32:
        case VR_INT64:
        case VR_FLOAT64:
        case VR_BOOL:
        case VR_DECIMAL128:
            break;
        case VR_UTF8:
            if (!k.offsets) return "a VR_UTF8 key needs its offsets";
            out.offsets = k.offsets;
            break;
        case VR_DICT32:
            if (!k.dictionary) return "a VR_DICT32 key needs its dictionary (the reference hashes the strings)";
            if (k.dictionary->size < 0) return "negative dictionary size";
            out.dict_size = k.dictionary->size;
            out.dict_hashes = hashes;
            break;
        default:
            return "unknown key lane";
    }
    return nullptr;
}
}  // namespace vr

extern "C" {

int vr_hash_dictionary(const vr_dictionary* dict, uint32_t* out_device, void* stream) {
    if (!dict || !out_device || dict->size < 0 || (dict->size > 0 && (!dict->offsets || !dict->data))) {
        t_last_error = "vr_hash_dictionary: null dictionary, output or buffers, or a negative size";
        return VR_ERR_INVALID;
    }
    cudaError_t e = launch_hash_dictionary(*dict, out_device, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        t_last_error = cudaGetErrorString(e);
        return VR_ERR_CUDA;
    }
    return VR_OK;
}

int vr_hash_rows(int32_t num_keys, const vr_column_type* types, const vr_column* keys, int64_t num_rows,
                 uint32_t* out_device, int32_t finish, void* stream) {
    if (num_keys < 0 || (num_keys > 0 && (!types || !keys)) || !out_device) {
        t_last_error = "vr_hash_rows: null descriptor or output pointer, or a negative key count";
        return VR_ERR_INVALID;
    }
    if (num_keys > kHashRowsScratchMaxKeys) {
        t_last_error = "vr_hash_rows: " + std::to_string(num_keys) + " key columns, at most " +
                       std::to_string(kHashRowsScratchMaxKeys);
        return VR_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // device memory: the descriptors, an error word, and the entry hashes of
    // dictionaries that come without them
    size_t bytes = 256 + sizeof(HashKey) * kHashRowsScratchMaxKeys;
    size_t dict_off[kHashRowsScratchMaxKeys] = {};
    for (int c = 0; c < num_keys; ++c) {
        if (types[c].lane == VR_DICT32 && keys[c].dictionary && !keys[c].dictionary->hashes) {
            dict_off[c] = bytes;
            bytes += ((size_t)std::max(0, keys[c].dictionary->size) * 4 + 255) & ~(size_t)255;
        }
    }
    char* mem = nullptr;
    cudaError_t e = cudaMalloc(&mem, bytes);
    if (e != cudaSuccess) {
        t_last_error = cudaGetErrorString(e);
        return VR_ERR_OOM;
    }
    uint32_t* bad = reinterpret_cast<uint32_t*>(mem);
    HashKey* kd = reinterpret_cast<HashKey*>(mem + 256);
    HashKey hk[kHashRowsScratchMaxKeys];
    int rc = VR_OK;
    for (int c = 0; c < num_keys && rc == VR_OK; ++c) {
        const uint32_t* hashes = nullptr;
        if (types[c].lane == VR_DICT32 && keys[c].dictionary) {
            hashes = keys[c].dictionary->hashes;
            if (!hashes) {
                hashes = reinterpret_cast<const uint32_t*>(mem + dict_off[c]);
                e = launch_hash_dictionary(*keys[c].dictionary, const_cast<uint32_t*>(hashes), st);
                if (e != cudaSuccess) rc = VR_ERR_CUDA;
            }
        }
        if (const char* why = hash_key_of(types[c], keys[c], hashes, hk[c])) {
            t_last_error = std::string("vr_hash_rows: ") + why;
            rc = VR_ERR_INVALID;
        }
    }
    uint32_t bad_host = 0;
    if (rc == VR_OK) {
        if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, 4, st);
        if (e == cudaSuccess && num_keys > 0) e = cudaMemcpyAsync(kd, hk, sizeof(HashKey) * num_keys, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = launch_hash_rows(num_keys, kd, num_rows, out_device, finish, bad, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&bad_host, bad, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            t_last_error = cudaGetErrorString(e);
            rc = VR_ERR_CUDA;
        } else if (bad_host) {
            t_last_error = "vr_hash_rows: a dictionary id lies outside its dictionary";
            rc = VR_ERR_INVALID;
        }
    } else {
        cudaStreamSynchronize(st);  // dictionary hashes already queued into `mem`
    }
    cudaFree(mem);
    return rc;
}

// The same kernel as vr_hash_rows with its descriptor table in the library's
// fixed device scratch instead of cudaMalloc'd memory. Meant for callers that
// must not allocate: cudaMalloc/cudaFree can synchronise the whole device
// (stalling a serving thread's other queries) and a memory-capped executor
// may have no device memory left to hand out. The scratch address is looked
// up once per device and kept; calls enqueue on `stream` and return.
int vr_hash_rows_noalloc(int32_t num_keys, const vr_column_type* types, const vr_column* keys, int64_t num_rows,
                         uint32_t* out_device, int32_t finish, void* stream) {
    if (num_keys < 0 || (num_keys > 0 && (!types || !keys)) || !out_device) {
        t_last_error = "vr_hash_rows_noalloc: null descriptor or output pointer, or a negative key count";
        return VR_ERR_INVALID;
    }
    if (num_keys > kHashRowsScratchMaxKeys) {
        t_last_error = "vr_hash_rows_noalloc: " + std::to_string(num_keys) + " key columns exceed its fixed scratch of " +
                       std::to_string(kHashRowsScratchMaxKeys);
        return VR_ERR_INVALID;
    }
    HashKey hk[kHashRowsScratchMaxKeys];
    for (int c = 0; c < num_keys; ++c) {
        const uint32_t* hashes = nullptr;
        if (types[c].lane == VR_DICT32 && keys[c].dictionary) {
            hashes = keys[c].dictionary->hashes;
            if (!hashes) {
                t_last_error = "vr_hash_rows_noalloc: a VR_DICT32 key must bring its dictionary's entry hashes "
                               "(vr_hash_dictionary)";
                return VR_ERR_INVALID;
            }
        }
        if (const char* why = hash_key_of(types[c], keys[c], hashes, hk[c])) {
            t_last_error = std::string("vr_hash_rows_noalloc: ") + why;
            return VR_ERR_INVALID;
        }
    }
    static std::mutex mu;
    static void* scratch_of[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess && (dev < 0 || dev >= 64)) {
        t_last_error = "vr_hash_rows_noalloc: device index above 63";
        return VR_ERR_UNSUPPORTED;
    }
    HashKey* kd = nullptr;
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> lk(mu);
        if (!scratch_of[dev]) {
            void* p = nullptr;
            e = hash_rows_scratch_address(&p);
            if (e == cudaSuccess) scratch_of[dev] = p;
        }
        kd = static_cast<HashKey*>(scratch_of[dev]);
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (e == cudaSuccess && num_keys > 0) e = cudaMemcpyAsync(kd, hk, sizeof(HashKey) * num_keys, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_hash_rows(num_keys, kd, num_rows, out_device, finish, nullptr, st);
    if (e != cudaSuccess) {
        t_last_error = cudaGetErrorString(e);
        return VR_ERR_CUDA;
    }
    return VR_OK;
}

int vr_jit_compile(const vr_agg_spec* spec, int32_t tier, int64_t* cubin_bytes, char* log, size_t cap) {
    return vr_jit_compile_shape(spec, tier, 256, 1, cubin_bytes, log, cap);
}

int vr_jit_compile_shape(const vr_agg_spec* spec, int32_t tier, int32_t threads, int32_t min_blocks,
                         int64_t* cubin_bytes, char* log, size_t cap) {
    if (!spec || threads < 32 || threads % 32 || threads > kMaxConsumerThreadsJit || min_blocks < 1) return VR_ERR_INVALID;
    Plan plan;
    int rc = compile_plan(*spec, plan);
    if (rc != VR_OK) {
        if (log && cap) std::snprintf(log, cap, "%s", plan.reason.c_str());
        return rc;
    }
    size_t bytes = 0;
    std::string err;
    JitShape shape;
    shape.kw = plan.prog.kw;
    shape.tier = tier == 0 ? kTierDirect : kTierHash;
    shape.rchunk = tier == 0 ? 4 : 1;
    shape.threads = threads;
    shape.min_blocks = min_blocks;
    bool ok = jit_compile_only(plan.prog, shape, &bytes, &err);
    if (log && cap) std::snprintf(log, cap, "%s", err.c_str());
    if (cubin_bytes) *cubin_bytes = (int64_t)bytes;
    return ok ? VR_OK : VR_ERR_UNSUPPORTED;
}

int vr_agg_plan(const vr_agg_spec* spec, vr_plan_info* info, vr_column_type* out_types, int32_t cap) {
    if (!spec || !info) return VR_ERR_INVALID;
    std::memset(info, 0, sizeof(*info));
    Plan plan;
    int rc = compile_plan(*spec, plan);
    std::snprintf(info->reason, sizeof(info->reason), "%s", plan.reason.c_str());
    if (rc != VR_OK) return rc;
    const Program& P = plan.prog;
    info->key_words = P.kw;
    info->acc_words = P.aw;
    info->slot_words = P.sw;
    info->num_ops = P.num_ops;
    info->num_outputs = plan.emit.num_out;
    info->staged_columns = P.num_cols;
    info->sentinel_layout = P.occ_word < 0 ? 1 : 0;
    info->direct_ok = plan.direct_ok ? 1 : 0;
    info->direct_slots = P.direct_slots;
    if (out_types)
        for (int i = 0; i < plan.emit.num_out && i < cap; ++i) out_types[i] = plan.out_types[i];
    return VR_OK;
}

}  // extern "C"
