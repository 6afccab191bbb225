// Grouped-aggregation kernels for sm_100a.
//
// k_aggregate is a persistent, warp-specialised kernel:
//   * one producer warp pulls tiles (instance, row range) from a global work
//     counter and stages every input column of the tile into shared memory
//     with bulk copies (cp.async.bulk, completion on an mbarrier), up to
//     `stages` tiles ahead;
//   * the consumer warps hash/probe and accumulate the staged rows:
//       direct tier - dictionary / boolean keys index a dense combination
//                     space; accumulators are thread-private in shared
//                     memory (no atomics), merged once per CTA at the end;
//       hash tier   - an open-addressing cache table in shared memory in
//                     front of the HBM table; rows whose key does not fit go
//                     straight to HBM (CAS insert + atomics). Optionally
//                     duplicate keys inside a warp are combined first
//                     (__match_any_sync + a tree over the peers).
// Replaces the per-row probe of GroupKeyTable (GroupKeyTable.java:709-764,
// 2296-2371) and the scatter loops of GroupedAccumulators
// (GroupedAccumulators.java:252-300, 424-472, 563-601, 852-862, 1052-1069).
#include <cub/device/device_select.cuh>
#include <cub/iterator/counting_input_iterator.cuh>

#include "agg_device.cuh"
#include "agg_kernels.cuh"

namespace vr {

// --------------------------------------------------------------- smem map
static __host__ __device__ inline int32_t align_up(int32_t x, int32_t a) { return (x + a - 1) / a * a; }

struct StageHdr {
    int64_t tile;  // -1: no more work
    int64_t row0;
    int32_t inst;
    int32_t rows;
    TileView view;
};

__host__ __device__ inline SmemMap smem_map_impl(int stages, int stage_bytes, int tier_bytes) {
    SmemMap m;
    m.prog = 0;
    m.desc = align_up((int32_t)sizeof(Program), 16);
    m.bars = align_up(m.desc + (int32_t)sizeof(BatchDesc), 16);
    m.hdr = align_up(m.bars + 2 * kMaxStages * 8, 16);
    m.stages = align_up(m.hdr + kMaxStages * (int32_t)sizeof(StageHdr), 128);
    m.tier = align_up(m.stages + stages * stage_bytes, 128);
    m.total = m.tier + tier_bytes;
    return m;
}
SmemMap smem_map(int stages, int stage_bytes, int tier_bytes) { return smem_map_impl(stages, stage_bytes, tier_bytes); }

VR_DEV void consumer_bar(int nt) { asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory"); }

VR_DEV void set_error(uint64_t* ctrl, uint64_t bits) { atomicOr((unsigned long long*)&ctrl[CTRL_ERROR], bits); }

// Copies n bytes (multiple of 8) global -> shared cooperatively.
VR_DEV void coop_copy(void* dst, const void* src, int bytes, int tid, int nt) {
    const uint64_t* s = reinterpret_cast<const uint64_t*>(src);
    uint64_t* d = reinterpret_cast<uint64_t*>(dst);
    for (int i = tid; i < bytes / 8; i += nt) d[i] = s[i];
}

// ------------------------------------------------------------ producer ---
// Locates the instance owning global tile t (descs sorted by tile_begin).
VR_DEV int find_instance(const BatchDesc* descs, int n, int64_t t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (descs[mid].tile_begin <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

VR_DEV void producer_loop(const Program& P, const BatchDesc* __restrict__ descs, const LaunchCfg& cfg,
                          uint64_t* tile_counter, uint64_t* full, uint64_t* empty, StageHdr* hdr,
                          unsigned char* stage0) {
    const int NS = cfg.stages;
    const int T = cfg.tile_rows;
    for (int64_t k = 0;; ++k) {
        int s = (int)(k % NS);
        uint32_t parity = (uint32_t)((k / NS) & 1);
        if (!mbar_wait(&empty[s], parity ^ 1u)) {
            set_error(descs[0].ctrl, kErrTimeout);
            return;
        }
        int64_t t = (int64_t)atomicAdd((unsigned long long*)tile_counter, 1ull);
        StageHdr& h = hdr[s];
        if (t >= cfg.total_tiles) {
            h.tile = -1;
            mbar_arrive(&full[s]);
            return;
        }
        int inst = cfg.num_desc == 1 ? 0 : find_instance(descs, cfg.num_desc, t);
        const BatchDesc& d = descs[inst];
        int64_t row0 = (t - d.tile_begin) * (int64_t)T;
        int64_t left = d.num_rows - row0;
        int rows = (int)(left < T ? left : T);
        h.tile = t;
        h.row0 = row0;
        h.inst = inst;
        h.rows = rows;
        unsigned char* st = stage0 + (size_t)s * cfg.lay.stage_bytes;
        bool bulk = d.tma && rows == T;
        uint32_t bytes = 0;
        for (int c = 0; c < P.num_cols; ++c) {
            int w = P.col_width[c];
            uint32_t db = w ? (uint32_t)(T * w) : (uint32_t)(T / 8);
            const char* src = d.col_data[c] + (w ? row0 * w : row0 / 8);
            h.view.data[c] = bulk ? (const char*)(st + cfg.lay.data_off[c]) : src;
            bytes += bulk ? db : 0;
            const uint32_t* vsrc = d.col_valid[c] ? d.col_valid[c] + row0 / 32 : nullptr;
            if (vsrc && cfg.lay.valid_off[c] >= 0 && bulk) {
                h.view.valid[c] = reinterpret_cast<const uint32_t*>(st + cfg.lay.valid_off[c]);
                bytes += (uint32_t)(T / 8);
            } else {
                h.view.valid[c] = vsrc;
            }
        }
        const uint32_t* ssrc = d.selection ? d.selection + row0 / 32 : nullptr;
        if (ssrc && cfg.lay.sel_off >= 0 && bulk) {
            h.view.sel = reinterpret_cast<const uint32_t*>(st + cfg.lay.sel_off);
            bytes += (uint32_t)(T / 8);
        } else {
            h.view.sel = ssrc;
        }
        if (bulk) {
            mbar_arrive_expect_tx(&full[s], bytes);
            for (int c = 0; c < P.num_cols; ++c) {
                int w = P.col_width[c];
                uint32_t db = w ? (uint32_t)(T * w) : (uint32_t)(T / 8);
                bulk_g2s(st + cfg.lay.data_off[c], d.col_data[c] + (w ? row0 * w : row0 / 8), db, &full[s]);
                if (d.col_valid[c] && cfg.lay.valid_off[c] >= 0)
                    bulk_g2s(st + cfg.lay.valid_off[c], d.col_valid[c] + row0 / 32, (uint32_t)(T / 8), &full[s]);
            }
            if (ssrc && cfg.lay.sel_off >= 0) bulk_g2s(st + cfg.lay.sel_off, ssrc, (uint32_t)(T / 8), &full[s]);
        } else {
            mbar_arrive(&full[s]);
        }
    }
}

// ------------------------------------------------------- row processing ---
VR_DEV void defer_row(const BatchDesc& D, int64_t row) {
    unsigned long long i = atomicAdd((unsigned long long*)&D.ctrl[CTRL_DEFERRED], 1ull);
    if ((int64_t)i < D.deferred_cap)
        D.deferred[i] = row;
    else
        set_error(D.ctrl, kErrDeferredFull);
}

// Hash tier: one warp-synchronous pass over up to 32 rows per warp. `r` is
// the lane's row in view coordinates; `live` says whether it holds a row.
template <int KW>
VR_DEV void hash_rows_pass(const Program& P, const BatchDesc& D, const TileView& v, int64_t r, bool live,
                           int64_t row_id, uint64_t* scache, int sslots, int s_probes, int g_probes,
                           bool warp_agg, uint32_t& new_groups) {
    const int lane = threadIdx.x & 31;
    uint64_t key[KW];
    bool side = false;
    uint64_t h = 0;
    if (live) {
        bool bad;
        pack_key<KW>(P, v, r, key, side, bad);
        if (bad) {
            set_error(D.ctrl, kErrBadKey);
            live = false;
        }
        h = hash_key<KW>(key);
    }
    if (!live) {
#pragma unroll
        for (int i = 0; i < KW; ++i) key[i] = 0;
    }
    uint32_t peers = 1u << lane;
    bool leader = live;
    PeerPlan pp;
    pp.steps = 0;
    pp.recv = 0;
    if (warp_agg) {
        uint32_t livemask = __ballot_sync(kFull, live);
        uint32_t m = kFull;
#pragma unroll
        for (int i = 0; i < KW; ++i) m &= __match_any_sync(kFull, (unsigned long long)key[i]);
        m &= live ? livemask : ~livemask;
        peers = m;
        leader = live && ((__ffs(peers) - 1) == lane);
        pp = make_peer_plan(peers, lane);
    }
    uint64_t* slot = nullptr;
    bool in_smem = false, defer = false;
    if (leader) {
        bool fresh = false, to = false;
        if (sslots > 0 && !side) {
            slot = find_or_insert<true, KW>(scache, sslots - 1, P.sw, key, h >> 32, false, s_probes, fresh, to);
            in_smem = slot != nullptr;
        }
        if (!slot) {
            slot = find_or_insert<false, KW>(D.table, D.cap_mask, P.sw, key, h, side, g_probes, fresh, to);
            if (slot && fresh) ++new_groups;
            if (to) set_error(D.ctrl, kErrLockTimeout);
            defer = (slot == nullptr) && !to;
        }
    }
    if (warp_agg) {
        uint32_t dm = __ballot_sync(kFull, defer);
        if (dm) defer = live && ((dm >> (__ffs(peers) - 1)) & 1u);
    }
    if (defer) defer_row(D, row_id);
    for (int i = 0; i < P.num_ops; ++i) {
        const OpDesc& o = P.ops[i];
        Contrib c;
        if (live) {
            op_contrib(o, v, r, c);
        } else {
#pragma unroll
            for (int j = 0; j < kMaxContrib; ++j) c.w[j] = 0;
        }
        if (warp_agg) peer_reduce(P, o, pp, c);
        if (slot) {
            if (in_smem)
                contrib_apply<true>(P, o, slot + P.kw + o.word, c);
            else
                contrib_apply<false>(P, o, slot + P.kw + o.word, c);
        }
    }
}

// Direct tier: thread-private accumulators, word (g, w) of consumer thread
// t at priv[(g * aw + w) * nt + t].
VR_DEV void direct_row(const Program& P, const BatchDesc& D, const TileView& v, int64_t r, uint64_t* priv, int nt,
                       int ctid) {
    int64_t g = direct_index(P, v, r);
    if (g < 0 || g >= P.direct_slots) {
        set_error(D.ctrl, kErrBadKey);
        return;
    }
    uint64_t* base = priv + (size_t)g * P.aw * nt + ctid;
    for (int i = 0; i < P.num_ops; ++i) {
        const OpDesc& o = P.ops[i];
        Contrib c;
        if (op_contrib(o, v, r, c) || o.kind == OP_COUNT_ROWS)
            contrib_apply_private(P, o, base + (size_t)o.word * nt, nt, c);
    }
}

// Applies one combined word pair (kind at word w) to global memory.
VR_DEV void word_apply_global(uint8_t kind, uint64_t* p, uint64_t a, uint64_t b) {
    switch (kind) {
        case WK_ADD:
            if (a) g_add(p, a);
            break;
        case WK_MAX:
            if (a) g_max(p, a);
            break;
        case WK_OR:
            if (a) g_or(p, a);
            break;
        case WK_F64: {
            if (a | b) {
                double s = __longlong_as_double((long long)a), cc = __longlong_as_double((long long)b);
                double old = g_fadd(reinterpret_cast<double*>(p), s);
                double nw, err;
                two_sum(old, s, nw, err);
                double tot = __dadd_rn(err, cc);
                if (tot != 0.0) g_fadd(reinterpret_cast<double*>(p + 1), tot);
            }
            break;
        }
        case WK_MAX128: {
            if (a | b) {
                uint64_t clo = ld_relaxed_g(p), chi = ld_relaxed_g(p + 1);
                for (int it = 0; it < 1 << 16 && u128_gt(a, b, clo, chi); ++it)
                    if (g_cas128(p, clo, chi, a, b)) break;
            }
            break;
        }
        default: break;
    }
}

// Direct tier flush: each consumer thread combines whole (group, word)
// columns of the private area and applies them to the dense HBM table.
VR_DEV void flush_direct(const Program& P, const BatchDesc& D, uint64_t* priv, int nt, int ctid) {
    const int64_t G = P.direct_slots;
    const int aw = P.aw;
    for (int64_t q = ctid; q < G * aw; q += nt) {
        int64_t g = q / aw;
        int w = (int)(q % aw);
        uint8_t kind = P.word_kind[w];
        if (kind == WK_F64C || kind == WK_MAX128L) continue;
        const uint64_t* col = priv + (size_t)q * nt;
        uint64_t a = 0, b = 0;
        switch (kind) {
            case WK_ADD:
                for (int t = 0; t < nt; ++t) a += col[t];
                break;
            case WK_MAX:
                for (int t = 0; t < nt; ++t) a = col[t] > a ? col[t] : a;
                break;
            case WK_OR:
                for (int t = 0; t < nt; ++t) a |= col[t];
                break;
            case WK_F64: {
                const uint64_t* col2 = col + nt;
                double s = 0.0, c = 0.0;
                for (int t = 0; t < nt; ++t)
                    dd_add(s, c, __longlong_as_double((long long)col[t]), __longlong_as_double((long long)col2[t]));
                a = (uint64_t)__double_as_longlong(s);
                b = (uint64_t)__double_as_longlong(c);
                break;
            }
            case WK_MAX128: {
                const uint64_t* col2 = col + nt;
                for (int t = 0; t < nt; ++t)
                    if (u128_gt(col[t], col2[t], a, b)) {
                        a = col[t];
                        b = col2[t];
                    }
                break;
            }
        }
        uint64_t* gslot = D.table + (size_t)g * P.sw;
        word_apply_global(kind, gslot + P.kw + w, a, b);
        if (w == 0 && a != 0) {  // COUNT_ROWS: the group exists, store its key (same bits from every CTA)
            uint64_t kbuf[kMaxKW];
            direct_key(P, g, kbuf);
            for (int i = 0; i < P.kw; ++i) gslot[i] = kbuf[i];
        }
    }
}

// Is slot occupied? Every live group has COUNT_ROWS (word 0) >= 1.
VR_DEV bool slot_used(const Program& P, const uint64_t* slot) { return slot[P.kw] != 0; }

// Merges one slot state (key + accumulators) into the HBM table of D.
// Returns false when the table had no room.
template <int KW>
VR_DEV bool merge_state(const Program& P, const BatchDesc& D, const uint64_t* src, uint32_t& new_groups,
                        int g_probes) {
    uint64_t key[KW];
#pragma unroll
    for (int i = 0; i < KW; ++i) key[i] = src[i];
    bool side = (P.occ_word < 0) && key[0] == 0;  // sentinel layout: stored 0 == the sentinel key
    bool fresh = false, to = false;
    uint64_t* slot = find_or_insert<false, KW>(D.table, D.cap_mask, P.sw, key, hash_key<KW>(key), side, g_probes,
                                               fresh, to);
    if (to) set_error(D.ctrl, kErrLockTimeout);
    if (!slot) return false;
    if (fresh) ++new_groups;
    for (int i = 0; i < P.num_ops; ++i) {
        const OpDesc& o = P.ops[i];
        Contrib c;
#pragma unroll
        for (int j = 0; j < kMaxContrib; ++j) c.w[j] = j < o.nwords ? src[KW + o.word + j] : 0;
        contrib_apply<false>(P, o, slot + KW + o.word, c);
    }
    return true;
}

// Hash tier flush: every occupied shared slot into HBM; slots HBM cannot
// take go to the spill list (merged by the host after the table grows).
template <int KW>
VR_DEV void flush_hash(const Program& P, const BatchDesc& D, uint64_t* scache, int sslots, int nt, int ctid,
                       uint32_t& new_groups, int g_probes) {
    for (int i = ctid; i < sslots; i += nt) {
        const uint64_t* s = scache + (size_t)i * P.sw;
        if (!slot_used(P, s)) continue;
        if (!merge_state<KW>(P, D, s, new_groups, g_probes)) {
            unsigned long long k = atomicAdd((unsigned long long*)&D.ctrl[CTRL_SPILLED], 1ull);
            if ((int64_t)k < D.spill_cap) {
                uint64_t* dst = D.spill + (size_t)k * P.sw;
                for (int w = 0; w < P.sw; ++w) dst[w] = s[w];
            } else {
                set_error(D.ctrl, kErrSpillFull);
            }
        }
    }
}

VR_DEV void zero_words(uint64_t* p, int64_t n, int tid, int nt) {
    for (int64_t i = tid; i < n; i += nt) p[i] = 0;
}

// ---------------------------------------------------------- the kernel ---
template <int KW, int TIER>
__global__ void __launch_bounds__(kMaxConsumerThreads + 32) k_aggregate(const BatchDesc* __restrict__ descs,
                                                                        const LaunchCfg cfg,
                                                                        uint64_t* __restrict__ tile_counter) {
    extern __shared__ __align__(128) unsigned char smem[];
    const SmemMap m = smem_map_impl(cfg.stages, cfg.lay.stage_bytes, cfg.tier_bytes);
    Program& P = *reinterpret_cast<Program*>(smem + m.prog);
    BatchDesc& D = *reinterpret_cast<BatchDesc*>(smem + m.desc);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + m.bars);
    uint64_t* empty = full + kMaxStages;
    StageHdr* hdr = reinterpret_cast<StageHdr*>(smem + m.hdr);
    unsigned char* stage0 = smem + m.stages;
    uint64_t* tier = reinterpret_cast<uint64_t*>(smem + m.tier);

    const int tid = threadIdx.x;
    const int NT = cfg.consumer_threads;
    coop_copy(&P, descs[0].prog, (int)sizeof(Program), tid, blockDim.x);
    if (tid == 0) {
        for (int s = 0; s < cfg.stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], (uint32_t)(NT / 32));
        }
    }
    __syncthreads();

    if (tid >= NT) {  // producer warp
        if (tid == NT) producer_loop(P, descs, cfg, tile_counter, full, empty, hdr, stage0);
        return;
    }

    // consumer warps
    const int ctid = tid;
    const int sslots = cfg.tier_bytes / (8 * P.sw);
    int cur = -1;
    uint32_t new_groups = 0;
    for (int64_t k = 0;; ++k) {
        int s = (int)(k % cfg.stages);
        uint32_t parity = (uint32_t)((k / cfg.stages) & 1);
        if (!mbar_wait(&full[s], parity)) {
            set_error(descs[0].ctrl, kErrTimeout);
            break;
        }
        const StageHdr& h = hdr[s];
        const int64_t tile = h.tile;
        if (tile < 0) break;
        const int inst = h.inst;
        if (inst != cur) {  // uniform across consumer warps: they all see every tile
            consumer_bar(NT);
            if (cur >= 0) {
                if (TIER == kTierDirect) {
                    flush_direct(P, D, tier, NT, ctid);
                } else {
                    flush_hash<KW>(P, D, tier, D.smem_slots < sslots ? D.smem_slots : sslots, NT, ctid, new_groups,
                                   cfg.g_probes);
                }
                if (new_groups) atomicAdd((unsigned long long*)&D.ctrl[CTRL_GROUPS], (unsigned long long)new_groups);
                new_groups = 0;
                consumer_bar(NT);
            }
            coop_copy(&D, &descs[inst], (int)sizeof(BatchDesc), ctid, NT);
            zero_words(tier, cfg.tier_bytes / 8, ctid, NT);
            consumer_bar(NT);
            cur = inst;
        }
        const TileView& v = h.view;
        const int rows = h.rows;
        const int64_t row0 = h.row0;
        if (TIER == kTierDirect) {
            for (int r = ctid; r < rows; r += NT) {
                if (v.sel && !bit_at(v.sel, r)) continue;
                direct_row(P, D, v, r, tier, NT, ctid);
            }
        } else {
            const int ss = D.smem_slots < sslots ? D.smem_slots : sslots;
            const bool wa = D.warp_agg != 0;
            for (int base = 0; base < rows; base += NT) {
                int r = base + ctid;
                bool live = r < rows && (v.sel == nullptr || bit_at(v.sel, r));
                hash_rows_pass<KW>(P, D, v, r, live, row0 + r, tier, ss, cfg.s_probes, cfg.g_probes, wa, new_groups);
            }
        }
        __syncwarp();
        if ((ctid & 31) == 0) mbar_arrive(&empty[s]);
    }
    if (cur >= 0) {
        consumer_bar(NT);
        if (TIER == kTierDirect) {
            flush_direct(P, D, tier, NT, ctid);
        } else {
            flush_hash<KW>(P, D, tier, D.smem_slots < sslots ? D.smem_slots : sslots, NT, ctid, new_groups,
                           cfg.g_probes);
        }
        if (new_groups) atomicAdd((unsigned long long*)&D.ctrl[CTRL_GROUPS], (unsigned long long)new_groups);
    }
}

// Deferred rows of one batch, against the HBM table only (rows are in batch
// coordinates; the view is the batch's own columns).
template <int KW>
__global__ void k_replay(const BatchDesc* __restrict__ desc, const int64_t* __restrict__ rows, int64_t n,
                         int g_probes) {
    __shared__ Program P;
    __shared__ BatchDesc D;
    coop_copy(&P, desc->prog, (int)sizeof(Program), threadIdx.x, blockDim.x);
    coop_copy(&D, desc, (int)sizeof(BatchDesc), threadIdx.x, blockDim.x);
    __syncthreads();
    TileView v;
    for (int c = 0; c < kMaxCols; ++c) {
        v.data[c] = D.col_data[c];
        v.valid[c] = D.col_valid[c];
    }
    v.sel = nullptr;
    uint32_t new_groups = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = (int64_t)blockIdx.x * blockDim.x;
    for (int64_t base = first; base < n; base += stride) {  // warp-uniform trip count
        int64_t i = base + threadIdx.x;
        bool live = i < n;
        int64_t r = live ? rows[i] : 0;
        hash_rows_pass<KW>(P, D, v, r, live, r, nullptr, 0, 0, g_probes, false, new_groups);
    }
    if (new_groups) atomicAdd((unsigned long long*)&D.ctrl[CTRL_GROUPS], (unsigned long long)new_groups);
}

// Merges slot states into the table of `desc` (rehash and spill merge).
template <int KW>
__global__ void k_merge_slots(const BatchDesc* __restrict__ desc, const uint64_t* __restrict__ src, int64_t n,
                              int g_probes) {
    __shared__ Program P;
    __shared__ BatchDesc D;
    coop_copy(&P, desc->prog, (int)sizeof(Program), threadIdx.x, blockDim.x);
    coop_copy(&D, desc, (int)sizeof(BatchDesc), threadIdx.x, blockDim.x);
    __syncthreads();
    uint32_t new_groups = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t* s = src + (size_t)i * P.sw;
        if (!slot_used(P, s)) continue;
        if (!merge_state<KW>(P, D, s, new_groups, g_probes)) set_error(D.ctrl, kErrSpillFull);
    }
    if (new_groups) atomicAdd((unsigned long long*)&D.ctrl[CTRL_GROUPS], (unsigned long long)new_groups);
}

// ------------------------------------------------------------- emission ---
struct Wide {  // signed 256-bit, little-endian limbs
    uint64_t l[4];
};
VR_DEV void wide_add_shifted(Wide& a, uint64_t x, bool x_signed, int shift_words32) {
    // adds x * 2^(32*shift) where x is a 64-bit (un)signed value
    uint64_t ext = (x_signed && (int64_t)x < 0) ? ~0ull : 0ull;
    uint64_t add[4] = {0, 0, 0, 0};
    // place x at bit offset 32*shift
    int bit = 32 * shift_words32;
    int w = bit / 64, b = bit % 64;
    uint64_t parts[5] = {0, 0, 0, 0, 0};
    if (b == 0) {
        parts[w] = x;
        for (int i = w + 1; i < 5; ++i) parts[i] = ext;
    } else {
        parts[w] = x << b;
        parts[w + 1] = (x >> (64 - b)) | (ext << b);
        for (int i = w + 2; i < 5; ++i) parts[i] = ext;
    }
    for (int i = 0; i < 4; ++i) add[i] = parts[i];
    unsigned __int128 carry = 0;
    for (int i = 0; i < 4; ++i) {
        unsigned __int128 s = (unsigned __int128)a.l[i] + add[i] + carry;
        a.l[i] = (uint64_t)s;
        carry = s >> 64;
    }
}
VR_DEV bool wide_fits_i128(const Wide& a) {
    uint64_t sign = ((int64_t)a.l[1] < 0) ? ~0ull : 0ull;
    return a.l[2] == sign && a.l[3] == sign;
}
// Exact total of a sum op's words (carry-save / limb representations).
VR_DEV Wide op_total(uint8_t op, const uint64_t* w, bool& overflow_flag) {
    Wide t = {{0, 0, 0, 0}};
    overflow_flag = false;
    switch (op) {
        case OP_SUM_I32:
            wide_add_shifted(t, w[0], true, 0);
            break;
        case OP_SUM_I64:
            wide_add_shifted(t, w[0], false, 0);
            wide_add_shifted(t, w[1], true, 1);
            break;
        case OP_SUM_D128:
        case OP_MERGE_DSUM:
        case OP_MERGE_DAVG:
            wide_add_shifted(t, w[0], false, 0);
            wide_add_shifted(t, w[1], false, 1);
            wide_add_shifted(t, w[2], false, 2);
            wide_add_shifted(t, w[3], true, 3);
            break;
        case OP_SUM_PROD:
            wide_add_shifted(t, w[0], false, 0);
            wide_add_shifted(t, w[1], true, 1);
            wide_add_shifted(t, w[2], false, 0);
            wide_add_shifted(t, w[3], false, 1);
            wide_add_shifted(t, w[4], false, 2);
            wide_add_shifted(t, w[5], true, 3);
            overflow_flag = false;  // rows past the product precision were nulled per row
            break;
    }
    return t;
}

VR_DEV double f64_total(const uint64_t* w) {
    double s = __longlong_as_double((long long)w[0]), c = __longlong_as_double((long long)w[1]);
    if (!isfinite(s)) return s;
    return __dadd_rn(s, c);
}

struct OutVal {
    uint64_t lo, hi;
    bool valid;
};

VR_DEV void emit_error(uint64_t* ctrl, int status) {
    atomicCAS((unsigned long long*)&ctrl[CTRL_EMIT_ERROR], 0ull, (unsigned long long)status);
}

VR_DEV OutVal out_value(const Program& P, const OutDesc& od, const uint64_t* slot, uint64_t* ctrl) {
    const uint64_t* acc = slot + P.kw;
    OutVal r = {0, 0, true};
    switch (od.kind) {
        case OUT_KEY: {
            const KeyField& kf = P.keys[od.key];
            if (kf.null_word >= 0 && ((slot[kf.null_word] >> kf.null_shift) & 1)) {
                r.valid = false;
                break;
            }
            uint64_t w = slot[kf.word];
            if (P.occ_word < 0) w ^= kSentinel;  // sentinel layout
            if (kf.bits == 64) {
                r.lo = w;
            } else if (kf.bits == 128) {
                r.lo = slot[kf.word];
                r.hi = slot[kf.word + 1];
            } else {
                uint64_t mask = kf.bits == 32 ? 0xffffffffull : ((1ull << kf.bits) - 1ull);
                r.lo = (w >> kf.shift) & mask;
            }
            break;
        }
        case OUT_COUNT:
            r.lo = acc[od.w0];
            break;
        case OUT_SUM_LONG:
        case OUT_SUM_LONG_NN: {
            if (od.kind == OUT_SUM_LONG && acc[od.w1] == 0) {
                r.valid = false;
                break;
            }
            bool of;
            Wide t = op_total(od.src_op, acc + od.w0, of);
            r.lo = t.l[0];
            if (od.flags & OUTF_CHECKED) {
                uint64_t sign = ((int64_t)t.l[0] < 0) ? ~0ull : 0ull;
                if (t.l[1] != sign || t.l[2] != sign || t.l[3] != sign) emit_error(ctrl, VR_ERR_OVERFLOW);
            }
            break;
        }
        case OUT_SUM_DOUBLE:
        case OUT_SUM_DOUBLE_NN: {
            if (od.kind == OUT_SUM_DOUBLE && acc[od.w1] == 0) {
                r.valid = false;
                break;
            }
            double d = f64_total(acc + od.w0);
            r.lo = (uint64_t)__double_as_longlong(d);
            break;
        }
        case OUT_MINMAX: {
            if (acc[od.w1] == 0) {
                r.valid = false;
                break;
            }
            uint64_t k = acc[od.w0];
            if (od.flags & OUTF_MIN) k = ~k;
            if (od.lane == VR_FLOAT64)
                r.lo = (uint64_t)__double_as_longlong(okey_f64_dec(k));
            else
                r.lo = (uint64_t)okey_i64_dec(k);
            break;
        }
        case OUT_MINMAX_D128: {
            if (acc[od.w1] == 0) {
                r.valid = false;
                break;
            }
            uint64_t lo = acc[od.w0], hi = acc[od.w0 + 1];
            if (od.flags & OUTF_MIN) {
                lo = ~lo;
                hi = ~hi;
            }
            r.lo = lo;
            r.hi = hi ^ 0x8000000000000000ull;
            break;
        }
        case OUT_DEC_SUM: {
            // WideDecimalSumAgg / WideDecimalAvgAgg buffers (VectorAggregates.scala:329-347, 374-389, 466-477)
            uint64_t cnt = acc[od.w1];
            if (od.src_op == OP_SUM_PROD && (acc[od.w0 + 6] & 1)) emit_error(ctrl, VR_ERR_DECIMAL_PRECISION);
            bool of;
            Wide t = op_total(od.src_op, acc + od.w0, of);
            if (cnt == 0) {
                if (od.flags & OUTF_FINAL) r.valid = false;  // empty group: null result
                break;                                      // buffer: zero
            }
            bool past = of || !wide_fits_i128(t) || !within_precision(t.l[0], (int64_t)t.l[1], od.precision);
            if (past) {
                r.valid = false;
                if ((od.flags & OUTF_FINAL) && !(od.flags & OUTF_NULL_ON_OVERFLOW))
                    emit_error(ctrl, VR_ERR_DECIMAL_PRECISION);
                break;
            }
            r.lo = t.l[0];
            r.hi = t.l[1];
            break;
        }
        case OUT_IS_EMPTY:
            if (od.flags & OUTF_FROM_FLAGS)
                r.lo = (acc[od.w1] & kFlagNonEmpty) ? 0 : 1;
            else
                r.lo = acc[od.w1] == 0 ? 1 : 0;
            break;
        case OUT_DEC_MERGE: {
            // WideDecimalSumMergeAgg.value / write (VectorAggregates.scala:727-766),
            // WideDecimalAvgMergeAgg.State.sum (VectorAggregates.scala:600-603)
            bool of;
            Wide t = op_total(od.src_op, acc + od.w0, of);
            uint64_t flags = acc[od.w0 + (od.src_op == OP_MERGE_DSUM ? 4 : 6)];
            bool non_empty = (flags & kFlagNonEmpty) != 0;
            bool overflowed = (flags & kFlagOverflow) != 0 || !wide_fits_i128(t);
            if (od.src_op == OP_MERGE_DSUM && !non_empty) {
                if (od.flags & OUTF_FINAL) r.valid = false;
                break;  // zero while empty
            }
            if (overflowed) {
                r.valid = false;
                if ((od.flags & OUTF_FINAL) && !(od.flags & OUTF_NULL_ON_OVERFLOW))
                    emit_error(ctrl, VR_ERR_DECIMAL_OVERFLOW);
                break;
            }
            if (!within_precision(t.l[0], (int64_t)t.l[1], od.precision)) {
                r.valid = false;
                if ((od.flags & OUTF_FINAL) && !(od.flags & OUTF_NULL_ON_OVERFLOW))
                    emit_error(ctrl, VR_ERR_DECIMAL_PRECISION);
                break;
            }
            r.lo = t.l[0];
            r.hi = t.l[1];
            break;
        }
        case OUT_MERGE_COUNT: {
            bool of;
            Wide t = op_total(OP_SUM_I64, acc + od.w0, of);
            r.lo = t.l[0];
            break;
        }
    }
    return r;
}

// Writes a bitmap of 32 rows per warp (bits of rows >= n are zero).
VR_DEV void write_bits(uint8_t* bm, int64_t o, int64_t n, bool bit) {
    uint32_t b = __ballot_sync(kFull, bit && o < n);
    const int lane = threadIdx.x & 31;
    int64_t base = o - lane;  // first row of this warp
    if (lane == 0 && base < n) {
        int64_t nbytes = (n + 7) / 8;
        int64_t byte0 = base / 8;
        for (int i = 0; i < 4 && byte0 + i < nbytes; ++i) bm[byte0 + i] = (uint8_t)(b >> (8 * i));
    }
}

__global__ void k_emit(const Program* __restrict__ prog, const EmitProgram* __restrict__ ep,
                       const uint64_t* __restrict__ table, const int64_t* __restrict__ slot_of, int64_t from,
                       int64_t to, const vr_out_column* __restrict__ outs, uint64_t* ctrl) {
    __shared__ Program P;
    __shared__ EmitProgram E;
    coop_copy(&P, prog, (int)sizeof(Program), threadIdx.x, blockDim.x);
    coop_copy(&E, ep, (int)sizeof(EmitProgram), threadIdx.x, blockDim.x);
    __syncthreads();
    const int64_t n = to - from;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        int64_t o = base + threadIdx.x;
        bool live = o < n;
        const uint64_t* slot = live ? table + (size_t)slot_of[from + o] * P.sw : nullptr;
        for (int j = 0; j < E.num_out; ++j) {
            const OutDesc& od = E.outs[j];
            OutVal v = {0, 0, false};
            if (live) v = out_value(P, od, slot, ctrl);
            write_bits(outs[j].validity, o, n, v.valid);
            switch (od.lane) {
                case VR_BOOL:
                    write_bits(reinterpret_cast<uint8_t*>(outs[j].data), o, n, v.valid && v.lo != 0);
                    break;
                case VR_INT32:
                case VR_DICT32:
                    if (live) reinterpret_cast<int32_t*>(outs[j].data)[o] = v.valid ? (int32_t)v.lo : 0;
                    break;
                case VR_INT64:
                case VR_FLOAT64:
                    if (live) reinterpret_cast<uint64_t*>(outs[j].data)[o] = v.valid ? v.lo : 0;
                    break;
                case VR_DECIMAL128:
                    if (live) {
                        reinterpret_cast<uint64_t*>(outs[j].data)[2 * o] = v.valid ? v.lo : 0;
                        reinterpret_cast<uint64_t*>(outs[j].data)[2 * o + 1] = v.valid ? v.hi : 0;
                    }
                    break;
            }
        }
    }
}

struct OccupiedPred {
    const uint64_t* table;
    int sw;
    int kw;
    __host__ __device__ bool operator()(const int64_t& i) const { return table[(size_t)i * sw + kw] != 0; }
};

// ------------------------------------------------------ reference hash ---
// HashKernels.mix32 / finish / fold / Decimal128.hash
// (kernels/src/main/java/io/vecruntime/kernels/HashKernels.java:51-64, 178-180;
//  Decimal128.java:155-160), Java int/long wrap-around arithmetic.
VR_DEV uint32_t jmix32(uint32_t h, uint32_t v) {
    h = (h ^ v) * 0x9E3779B1u;
    return h ^ (h >> 15);
}
VR_DEV uint32_t jfinish(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}
VR_DEV uint32_t jfold(uint64_t v) { return (uint32_t)(v ^ (v >> 32)); }
VR_DEV uint64_t jdec_hash(uint64_t hi, uint64_t lo) {
    uint64_t h = lo * 0x9E3779B97F4A7C15ull;
    h ^= (h >> 32) ^ (hi * 0xC2B2AE3D27D4EB4Full);
    h ^= h >> 29;
    return h;
}

__global__ void k_hash_rows(int nk, const vr_column_type* __restrict__ types, const vr_column* __restrict__ keys,
                            int64_t n, uint32_t* __restrict__ out, int finish) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t h = 0x2545F491u;
        for (int c = 0; c < nk; ++c) {
            const vr_column& col = keys[c];
            bool valid = col.validity == nullptr || ((col.validity[i >> 3] >> (i & 7)) & 1);
            uint32_t v;
            if (!valid) {
                v = 0x7F4A7C15u;
            } else {
                switch (types[c].lane) {
                    case VR_INT32:
                    case VR_DICT32:
                        v = (uint32_t) reinterpret_cast<const int32_t*>(col.data)[i];
                        break;
                    case VR_INT64:
                    case VR_FLOAT64:
                        v = jfold(reinterpret_cast<const uint64_t*>(col.data)[i]);
                        break;
                    case VR_BOOL:
                        v = (reinterpret_cast<const uint8_t*>(col.data)[i >> 3] >> (i & 7)) & 1;
                        break;
                    case VR_DECIMAL128: {
                        const uint64_t* p = reinterpret_cast<const uint64_t*>(col.data) + 2 * i;
                        v = jfold(jdec_hash(p[1], p[0]));
                        break;
                    }
                    default:
                        v = 0;
                }
            }
            h = jmix32(h, v);
        }
        out[i] = finish ? jfinish(h) : h;
    }
}

// ------------------------------------------------------------ launchers ---
template <int KW, int TIER>
static cudaError_t launch_agg_t(const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                                cudaStream_t stream) {
    auto fn = k_aggregate<KW, TIER>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, cfg.smem_bytes);
    if (e != cudaSuccess) return e;
    fn<<<blocks, cfg.consumer_threads + 32, cfg.smem_bytes, stream>>>(descs, cfg, tile_counter);
    return cudaGetLastError();
}

cudaError_t launch_aggregate(int kw, int tier, const BatchDesc* descs, const LaunchCfg& cfg, int blocks,
                             uint64_t* tile_counter, cudaStream_t stream) {
    if (tier == kTierDirect) {
        switch (kw) {
            case 1: return launch_agg_t<1, kTierDirect>(descs, cfg, blocks, tile_counter, stream);
            case 2: return launch_agg_t<2, kTierDirect>(descs, cfg, blocks, tile_counter, stream);
            case 3: return launch_agg_t<3, kTierDirect>(descs, cfg, blocks, tile_counter, stream);
            case 4: return launch_agg_t<4, kTierDirect>(descs, cfg, blocks, tile_counter, stream);
        }
    } else {
        switch (kw) {
            case 1: return launch_agg_t<1, kTierHash>(descs, cfg, blocks, tile_counter, stream);
            case 2: return launch_agg_t<2, kTierHash>(descs, cfg, blocks, tile_counter, stream);
            case 3: return launch_agg_t<3, kTierHash>(descs, cfg, blocks, tile_counter, stream);
            case 4: return launch_agg_t<4, kTierHash>(descs, cfg, blocks, tile_counter, stream);
        }
    }
    return cudaErrorInvalidValue;
}

static int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return (int)b;
}

cudaError_t launch_replay(int kw, const BatchDesc* desc, const int64_t* rows, int64_t n, int g_probes,
                          cudaStream_t stream) {
    int b = grid_for(n, 256);
    switch (kw) {
        case 1: k_replay<1><<<b, 256, 0, stream>>>(desc, rows, n, g_probes); break;
        case 2: k_replay<2><<<b, 256, 0, stream>>>(desc, rows, n, g_probes); break;
        case 3: k_replay<3><<<b, 256, 0, stream>>>(desc, rows, n, g_probes); break;
        case 4: k_replay<4><<<b, 256, 0, stream>>>(desc, rows, n, g_probes); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_merge_slots(int kw, const BatchDesc* desc, const uint64_t* slots, int64_t n, int g_probes,
                               cudaStream_t stream) {
    int b = grid_for(n, 256);
    switch (kw) {
        case 1: k_merge_slots<1><<<b, 256, 0, stream>>>(desc, slots, n, g_probes); break;
        case 2: k_merge_slots<2><<<b, 256, 0, stream>>>(desc, slots, n, g_probes); break;
        case 3: k_merge_slots<3><<<b, 256, 0, stream>>>(desc, slots, n, g_probes); break;
        case 4: k_merge_slots<4><<<b, 256, 0, stream>>>(desc, slots, n, g_probes); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_compact_kw(int kw, const uint64_t* table, int64_t slots, int sw, int64_t* out, int64_t* num_dev,
                              void* temp, size_t* temp_bytes, cudaStream_t stream) {
    OccupiedPred pred;
    pred.table = table;
    pred.sw = sw;
    pred.kw = kw;
    cub::CountingInputIterator<int64_t> it(0);
    return cub::DeviceSelect::If(temp, *temp_bytes, it, out, num_dev, slots, pred, stream);
}

cudaError_t launch_emit(const Program* prog_dev, const EmitProgram* emit_dev, const uint64_t* table,
                        const int64_t* slot_of, int64_t from, int64_t to, const vr_out_column* outs_dev,
                        uint64_t* ctrl, cudaStream_t stream) {
    int64_t n = to - from;
    if (n <= 0) return cudaSuccess;
    int b = grid_for(n, 256);
    k_emit<<<b, 256, 0, stream>>>(prog_dev, emit_dev, table, slot_of, from, to, outs_dev, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_hash_rows(int num_keys, const vr_column_type* types_dev, const vr_column* keys_dev, int64_t n,
                             uint32_t* out, int finish, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    k_hash_rows<<<grid_for(n, 256), 256, 0, stream>>>(num_keys, types_dev, keys_dev, n, out, finish);
    return cudaGetLastError();
}

cudaError_t upload_pow10() {
    uint64_t lo[39], hi[39];
    unsigned __int128 v = 1;
    for (int i = 0; i < 39; ++i) {
        lo[i] = (uint64_t)v;
        hi[i] = (uint64_t)(v >> 64);
        v *= 10;
    }
    cudaError_t e = cudaMemcpyToSymbol(c_pow10_lo, lo, sizeof(lo));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_pow10_hi, hi, sizeof(hi));
}

}  // namespace vr
