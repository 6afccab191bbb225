// Runtime state behind the C ABI: the aggregate handle, its device table,
// staging, and the launch configuration. Shared by abi.cu, batched.cu,
// tune.cpp and serving.cpp.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <unordered_map>
#include <vector>

#include "agg_kernels.cuh"
#include "plan.h"
#include "vrgpu.h"

namespace vr {

// Launch configuration of one handle (chosen by the tuner or forced).
struct Config {
    int tier = kTierHash;
    int warp_agg = 0;
    int threads = 256;        // consumer threads
    int blocks_per_sm = 1;
    int tile_rows = 2048;
    int rchunk = 4;           // rows per consumer thread per chunk
    int stages = 2;
    int smem_slots = 0;       // hash tier shared cache
    int tma = 1;
    int g_probes = 512;
    int s_probes = 8;
    int64_t capacity = 0;     // HBM table slots (hash tier: power of two)
};

// One staging set: a batch in flight (ping-pong between two).
struct StageSlot {
    char* dev = nullptr;        // staged host columns
    size_t dev_cap = 0;
    BatchDesc* desc_host = nullptr;  // pinned
    BatchDesc* desc_dev = nullptr;
    uint64_t* ctrl_dev = nullptr;
    uint64_t* ctrl_host = nullptr;   // pinned mirror, copied after each launch
    int64_t* deferred = nullptr;
    int64_t* deferred_tmp = nullptr;
    int64_t deferred_cap = 0;
    uint64_t* spill = nullptr;
    int64_t spill_cap = 0;
    cudaEvent_t done = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;  // kernel timing (trace)
    cudaEvent_t h0 = nullptr;                // H2D start (trace)
    cudaEvent_t copied = nullptr;            // this slot's H2D copies are done
    bool pending_done_recorded = false;      // `done` has been recorded at least once
    BatchDesc launched{};             // host copy of the last launch's descriptor
    bool pending = false;
    bool timed = false;
    bool staged_h2d = false;
    int64_t rows = 0;
    int32_t* remap_dev = nullptr;   // batch dictionary -> table id maps of this batch
    int32_t* remap_host = nullptr;  // pinned staging of those maps
    int64_t remap_cap = 0;          // entries of both
};

// The strings of one VR_COL_BATCH_DICTIONARY key, in table-id order, and
// their ids: every batch's dictionary is mapped onto it (GroupKeyTable's
// StringDictionary, GroupKeyTable.java:1308-1430).
// A table dictionary's string -> id map: open addressing over the strings'
// bytes kept in one arena, so mapping a batch's dictionary (once per batch,
// often right after a reset) allocates nothing per entry. It offers what the
// batch mapping uses of a std::unordered_map: find / end / emplace / size /
// clear, an entry reached as `it->second`, valid until the next emplace.
class StrIdMap {
public:
    struct Entry {
        int32_t second;
    };
    Entry* find(const std::string& s) {
        if (slots_.empty()) return nullptr;
        const uint64_t h = hash(s.data(), s.size());
        for (size_t i = h & (slots_.size() - 1);; i = (i + 1) & (slots_.size() - 1)) {
            const int32_t e = slots_[i];
            if (e < 0) return nullptr;
            if (hashes_[e] == h && len_[e] == s.size() && std::memcmp(arena_.data() + off_[e], s.data(), s.size()) == 0)
                return &vals_[e];
        }
    }
    Entry* end() { return nullptr; }
    std::pair<Entry*, bool> emplace(const std::string& s, int32_t id) {
        if (Entry* e = find(s)) return {e, false};
        if (2 * (vals_.size() + 1) > slots_.size()) grow();
        const uint64_t h = hash(s.data(), s.size());
        const int32_t e = (int32_t)vals_.size();
        off_.push_back(arena_.size());
        len_.push_back(s.size());
        hashes_.push_back(h);
        vals_.push_back(Entry{id});
        arena_.append(s);
        size_t i = h & (slots_.size() - 1);
        while (slots_[i] >= 0) i = (i + 1) & (slots_.size() - 1);
        slots_[i] = e;
        return {&vals_[e], true};
    }
    size_t size() const { return vals_.size(); }
    void clear() {
        std::fill(slots_.begin(), slots_.end(), -1);
        arena_.clear();
        off_.clear();
        len_.clear();
        hashes_.clear();
        vals_.clear();
    }

private:
    static uint64_t hash(const char* p, size_t n) {
        uint64_t h = 0x9E3779B97F4A7C15ull ^ (n * 0xFF51AFD7ED558CCDull);
        size_t i = 0;
        for (; i + 8 <= n; i += 8) {
            uint64_t w;
            std::memcpy(&w, p + i, 8);
            h = (h ^ w) * 0xC4CEB9FE1A85EC53ull;
            h ^= h >> 29;
        }
        uint64_t t = 0;
        std::memcpy(&t, p + i, n - i);
        h = (h ^ t) * 0xC4CEB9FE1A85EC53ull;
        return h ^ (h >> 32);
    }
    void grow() {
        const size_t cap = slots_.empty() ? 1024 : 2 * slots_.size();
        slots_.assign(cap, -1);
        for (int32_t e = 0; e < (int32_t)vals_.size(); ++e) {
            size_t i = hashes_[e] & (cap - 1);
            while (slots_[i] >= 0) i = (i + 1) & (cap - 1);
            slots_[i] = e;
        }
    }
    std::vector<int32_t> slots_;
    std::string arena_;
    std::vector<size_t> off_, len_;
    std::vector<uint64_t> hashes_;
    std::vector<Entry> vals_;
};

struct TableDict {
    int key = -1;                  // key index in the spec
    int32_t limit = 0;             // the declared dict_size (0: no limit)
    StrIdMap ids;
    std::vector<int32_t> offsets{0};
    std::string bytes;
};

struct JitKernel;

struct DeviceInfo {
    int sms = 148;
    int smem_optin = 232448;     // per block
    int smem_per_sm = 233472;
    int smem_reserved = 1024;    // per block, by the system
    bool ready = false;
    // Whether `blocks` CTAs of `smem` dynamic shared bytes fit on one SM.
    bool fits(int blocks, int smem) const { return blocks * (smem + smem_reserved) <= smem_per_sm; }
};
DeviceInfo& device_info(int device);

}  // namespace vr

struct vr_agg {
    int device = 0;
    cudaStream_t stream = nullptr;       // kernels, emission
    cudaStream_t copy_stream = nullptr;  // host -> device staging copies
    bool own_stream = false;
    // spec copy
    std::vector<vr_column_type> columns;
    std::vector<int32_t> keys;
    std::vector<vr_agg_fn> fns;
    vr_agg_spec spec{};
    vr::Plan plan;
    vr::Config cfg;
    vr::LaunchCfg launch{};
    int blocks = 0;
    vr::Program* prog_dev = nullptr;
    vr::EmitProgram* emit_dev = nullptr;
    uint64_t* table = nullptr;
    int64_t table_slots = 0;      // slots scanned by compaction (incl. the side slot)
    vr::StageSlot slot[2];
    int next_slot = 0;
    int64_t groups_known = 0;
    bool clear_queued = false;  // vr_agg_reset's memset may still be in flight on `stream`
    // compaction / emission
    bool compact_valid = false;
    int64_t* slot_of = nullptr;
    int64_t slot_of_cap = 0;
    int64_t* num_dev = nullptr;
    int64_t num_groups = 0;
    void* cub_temp = nullptr;
    size_t cub_temp_bytes = 0;
    vr_out_column* outs_dev = nullptr;
    vr_out_column* outs_host = nullptr;  // pinned
    char* emit_stage = nullptr;
    size_t emit_stage_cap = 0;
    uint64_t* emit_ctrl = nullptr;       // pinned mirror word
    // descriptor + control block for rehash / emission (never a batch's)
    vr::BatchDesc* aux_desc_host = nullptr;  // pinned
    vr::BatchDesc* aux_desc_dev = nullptr;
    uint64_t* aux_ctrl_dev = nullptr;
    uint64_t* aux_ctrl_host = nullptr;       // pinned
    // status
    int status = VR_OK;
    std::string last_error;
    vr_agg_stats stats{};
    bool trace = false;
    bool dead = false;
    vr::JitKernel* jit = nullptr;  // the spec's own kernel (owned by the process-wide cache)
    bool prebuilt_only = false;    // no per-spec kernel: blocks stay within the prebuilt kernel's bounds
    std::string jit_error;         // why it could not be compiled, when it could not
    std::vector<vr::TableDict> tdicts;  // one per VR_COL_BATCH_DICTIONARY key
};

namespace vr {
// shared helpers (abi.cu)
int set_err(vr_agg* h, int code, const std::string& msg);
int cuda_err(vr_agg* h, cudaError_t e, const char* what);
int agg_build(const vr_agg_spec* spec, const vr_tune_choice* forced, vr_agg** out, cudaStream_t stream);
// Fills a BatchDesc for a device-resident batch (no copies).
void fill_desc(vr_agg* h, const vr_batch& b, BatchDesc& d, uint64_t* ctrl, const StageSlot& s, int64_t tile_begin);
int agg_resolve_all(vr_agg* h);
// Staging and deferred-row lists sized now for batches of up to `rows` rows.
int agg_reserve(vr_agg* h, int64_t rows);
cudaError_t agg_launch(vr_agg* h, const BatchDesc* descs, const LaunchCfg& L, int blocks, uint64_t* tile_counter,
                       cudaStream_t st);
int64_t tiles_for(const vr_agg* h, int64_t rows);
// Bytes of one pipeline stage of T rows, and where each column lands in it.
int32_t stage_bytes_for(const Program& P, int T);
void fill_layout(const Program& P, int T, StageLayout& L);
// CTAs of `threads` consumer threads (plus the producer warp), `smem` dynamic
// shared bytes and `regs` registers per thread (0: unknown) that fit one SM, at most `want`.
int ctas_per_sm(const DeviceInfo& di, int smem, int regs, int threads, int want);
int64_t next_pow2(int64_t x);
// Why a batch breaks the spec's nullability (a bitmap on a non-nullable column), or null.
const char* batch_nullability_error(const vr_agg* h, const vr_batch& b);
void set_thread_error(const std::string& msg);
}  // namespace vr
