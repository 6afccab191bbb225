// Autotuner (see tune.h). Entries live in a process-wide map and can be saved
// to / loaded from a text file (spark.vecruntime.agg.gpu.autotuneCache).
// vr_tune_search measures candidates on a real batch with CUDA events.
#include "tune.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace vr {

namespace {

struct Entry {
    vr_tune_choice choice;
    double rows_per_s;
};

std::mutex g_mu;
std::map<std::tuple<uint64_t, int, int>, Entry> g_table;

int log2_bucket(int64_t x) {
    int b = 0;
    while (x > 1) {
        x >>= 1;
        ++b;
    }
    return b;
}

uint64_t fnv(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) {
        h ^= (v >> (8 * i)) & 0xff;
        h *= 0x100000001b3ull;
    }
    return h;
}

}  // namespace

// Everything in a spec that changes the kernel or its cost: column lanes,
// nullability, dictionary sizes, decimal types and flags, the keys, and every
// function field (kind, inputs, flags, types, product terms and precision).
uint64_t spec_signature(const vr_agg_spec& s) {
    uint64_t h = 0xcbf29ce484222325ull;
    h = fnv(h, (uint64_t)s.num_columns);
    for (int c = 0; c < s.num_columns; ++c) {
        const vr_column_type& t = s.columns[c];
        h = fnv(h, (uint64_t)t.lane | ((uint64_t)t.nullable << 8) | ((uint64_t)(uint32_t)t.dict_size << 16));
        h = fnv(h, (uint64_t)(uint32_t)t.precision | ((uint64_t)(uint32_t)t.scale << 16) | ((uint64_t)(uint32_t)t.flags << 32));
    }
    for (int k = 0; k < s.num_keys; ++k) h = fnv(h, (uint64_t)s.key_columns[k] + 1000);
    for (int f = 0; f < s.num_fns; ++f) {
        const vr_agg_fn& fn = s.fns[f];
        h = fnv(h, (uint64_t)fn.kind | ((uint64_t)(uint32_t)fn.input << 8) | ((uint64_t)(uint32_t)fn.input2 << 24) |
                       ((uint64_t)fn.num_terms << 40));
        h = fnv(h, (uint64_t)(uint32_t)fn.flags | ((uint64_t)(uint32_t)fn.precision << 16) |
                       ((uint64_t)(uint32_t)fn.scale << 32) | ((uint64_t)(uint32_t)fn.product_precision << 48));
        h = fnv(h, (uint64_t)(uint32_t)fn.result_precision | ((uint64_t)(uint32_t)fn.result_scale << 32));
        for (int t = 0; t < fn.num_terms && t < 3; ++t)
            h = fnv(h, ((uint64_t)(uint32_t)fn.terms[t].column | ((uint64_t)(uint32_t)fn.terms[t].sign << 32)) ^
                           (uint64_t)fn.terms[t].addend);
    }
    return h;
}

static std::tuple<uint64_t, int, int> key_of(const vr_agg_spec& s, int64_t rows) {
    return std::make_tuple(spec_signature(s), log2_bucket(rows > 0 ? rows : 1),
                           log2_bucket(s.est_groups > 0 ? s.est_groups : 1));
}

bool tune_lookup_internal(const vr_agg_spec& spec, int64_t rows, vr_tune_choice* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_table.find(key_of(spec, rows));
    if (it == g_table.end()) return false;
    *out = it->second.choice;
    return true;
}

}  // namespace vr

using namespace vr;

extern "C" {

int vr_tune_lookup(const vr_agg_spec* spec, int64_t rows, vr_tune_choice* out) {
    if (!spec || !out) return 0;
    return tune_lookup_internal(*spec, rows, out) ? 1 : 0;
}

int vr_tune_record(const vr_agg_spec* spec, int64_t rows, const vr_tune_choice* choice, double rows_per_s) {
    if (!spec || !choice) return VR_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_mu);
    auto k = key_of(*spec, rows);
    auto it = g_table.find(k);
    if (it == g_table.end() || rows_per_s > it->second.rows_per_s) g_table[k] = Entry{*choice, rows_per_s};
    return VR_OK;
}

int vr_tune_save(const char* path) {
    if (!path) return VR_ERR_INVALID;
    std::FILE* f = std::fopen(path, "w");
    if (!f) return VR_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_mu);
    std::fprintf(f, "# vrgpu autotune v1: signature rows_log2 groups_log2 tier warp_agg threads bps tile smem cap rows_per_s\n");
    for (auto& kv : g_table) {
        const vr_tune_choice& c = kv.second.choice;
        std::fprintf(f, "%llu %d %d %d %d %d %d %d %d %lld %.6g\n", (unsigned long long)std::get<0>(kv.first),
                     std::get<1>(kv.first), std::get<2>(kv.first), c.tier, c.warp_agg, c.threads, c.blocks_per_sm,
                     c.tile_rows, c.smem_slots, (long long)c.table_capacity, kv.second.rows_per_s);
    }
    std::fclose(f);
    return VR_OK;
}

int vr_tune_load(const char* path) {
    if (!path) return VR_ERR_INVALID;
    std::FILE* f = std::fopen(path, "r");
    if (!f) return VR_ERR_INVALID;
    char line[512];
    std::lock_guard<std::mutex> lk(g_mu);
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#') continue;
        unsigned long long sig;
        int rb, gb;
        vr_tune_choice c;
        std::memset(&c, 0, sizeof(c));
        long long cap;
        double rps;
        if (std::sscanf(line, "%llu %d %d %d %d %d %d %d %d %lld %lf", &sig, &rb, &gb, &c.tier, &c.warp_agg, &c.threads,
                        &c.blocks_per_sm, &c.tile_rows, &c.smem_slots, &cap, &rps) == 11) {
            c.table_capacity = cap;
            g_table[std::make_tuple((uint64_t)sig, rb, gb)] = Entry{c, rps};
        }
    }
    std::fclose(f);
    return VR_OK;
}

int vr_tune_search(const vr_agg_spec* spec, const vr_batch* batch, int32_t iters, vr_tune_choice* best,
                   double* best_rps) {
    if (!spec || !batch || batch->location != VR_DEVICE || !best) return VR_ERR_INVALID;
    if (iters < 1) iters = 3;
    vr_plan_info info;
    if (vr_agg_plan(spec, &info, nullptr, 0) != VR_OK) return VR_ERR_UNSUPPORTED;
    std::vector<vr_tune_choice> cands;
    auto add = [&](int tier, int wa, int threads, int tile, int smem, int ctas) {
        vr_tune_choice c;
        std::memset(&c, 0, sizeof(c));
        c.tier = tier;
        c.warp_agg = wa;
        c.threads = threads;
        c.tile_rows = tile;
        c.smem_slots = smem;
        c.blocks_per_sm = ctas;
        cands.push_back(c);
    };
    // direct tier: threads x tile x CTAs per SM around the measured best
    // (two CTAs of 160 threads with 640-row tiles on the decimal report)
    if (info.direct_ok) {
        const int shapes[][3] = {{160, 640, 2}, {128, 512, 2}, {96, 384, 3}, {64, 256, 4}, {256, 1024, 1}};
        for (const auto& sh : shapes) add(0, 0, sh[0], sh[1], 0, sh[2]);
    }
    // hash tiers: the default shape (whole table in shared memory when it
    // fits, else a cache sized to the batch), hot-key caches from 256 to
    // 1,024 slots with tiles from 1,024 down to 256 rows, and HBM only
    for (int wa : {0, 1}) {
        add(1, wa, 0, 0, 0, 0);
        for (int tile : {1024, 512, 256})
            for (int slots : {256, 512, 1024}) add(1, wa, 256, tile, slots, 2);
        // one CTA per SM of 512 threads: room for a 2,048 or 4,096-slot cache
        // (more of a skewed key's head in shared memory)
        for (int slots : {2048, 4096}) add(1, wa, 512, 512, slots, 1);
        add(2, wa, 256, 1024, 0, 2);
    }
    double best_v = -1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (auto& c : cands) {
        vr_agg* h = nullptr;
        if (vr_agg_create_tuned(spec, &c, &h) != VR_OK) continue;
        cudaStream_t st = (cudaStream_t)vr_agg_stream(h);
        bool ok = vr_agg_update(h, batch) == VR_OK && vr_agg_sync(h) == VR_OK;  // warm-up
        float total = 0;
        for (int i = 0; ok && i < iters; ++i) {
            ok = vr_agg_reset(h) == VR_OK;
            cudaEventRecord(e0, st);
            ok = ok && vr_agg_update(h, batch) == VR_OK;
            cudaEventRecord(e1, st);
            ok = ok && vr_agg_sync(h) == VR_OK;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            total += ms;
        }
        vr_agg_destroy(h);
        if (!ok || total <= 0) continue;
        double rps = (double)batch->num_rows * iters / (total * 1e-3);
        if (rps > best_v) {
            best_v = rps;
            *best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_v < 0) return VR_ERR_UNSUPPORTED;
    if (best_rps) *best_rps = best_v;
    return vr_tune_record(spec, batch->num_rows, best, best_v);
}

}  // extern "C"
