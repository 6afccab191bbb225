// The aggregate kernel body and its helpers (device code only). Included by
// the ahead-of-time kernels (agg_kernels.cu) and by the per-spec kernels
// compiled at run time with NVRTC (jit.cpp), where VR_JIT is defined and the
// Program is a compile-time constant: every loop over ops and key fields then
// unrolls into straight-line code for that spec.
#pragma once
#include "agg_device.cuh"
#include "agg_types.h"

namespace vr {

// --------------------------------------------------------------- smem map
static __host__ __device__ inline int32_t align_up(int32_t x, int32_t a) { return (x + a - 1) / a * a; }

struct StageHdr {
    int64_t tile;  // -1: no more work
    int64_t row0;
    int32_t inst;
    int32_t rows;
    int32_t staged;  // 1: the tile's column data was bulk-copied into the stage
    int32_t pad_;
    TileView view;
};

__host__ __device__ inline SmemMap smem_map_impl(int stages, int stage_bytes, int tier_bytes) {
    SmemMap m;
    m.prog = 0;
    m.desc = align_up((int32_t)sizeof(Program), 16);
    m.pdesc = align_up(m.desc + (int32_t)sizeof(BatchDesc), 16);  // the producer's own copy
    m.bars = align_up(m.pdesc + (int32_t)sizeof(BatchDesc), 16);
    m.hdr = align_up(m.bars + 2 * kMaxStages * 8, 16);
    m.stages = align_up(m.hdr + kMaxStages * (int32_t)sizeof(StageHdr), 128);
    m.tier = align_up(m.stages + stages * stage_bytes, 128);
    m.total = m.tier + tier_bytes;
    return m;
}

VR_DEV void consumer_bar(int nt) { asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory"); }

VR_DEV void set_error(uint64_t* ctrl, uint64_t bits) { atomicOr((unsigned long long*)&ctrl[CTRL_ERROR], bits); }

// Copies n bytes (multiple of 8) global -> shared cooperatively.
VR_DEV void coop_copy(void* dst, const void* src, int bytes, int tid, int nt) {
    const uint64_t* s = reinterpret_cast<const uint64_t*>(src);
    uint64_t* d = reinterpret_cast<uint64_t*>(dst);
    #pragma unroll 1  // once per CTA: keep it small
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

// The producer thread: takes tiles from the work counter in runs of
// cfg.tile_run consecutive tiles (the next run is fetched while the last tile
// of the current one is issued, so the atomic's round trip overlaps it),
// finds the tile's instance with a
// cursor that only moves forward (a producer's tile indices only grow), keeps
// that instance's descriptor in its own shared-memory copy (reloaded only
// when the instance changes), and issues the tile's bulk copies.
VR_DEV void producer_loop(const Program& P, const BatchDesc* __restrict__ descs, const LaunchCfg& cfg,
                          uint64_t* tile_counter, uint64_t* full, uint64_t* empty, StageHdr* hdr,
                          unsigned char* stage0, BatchDesc* pd) {
    const int NS = cfg.stages;
    const int T = cfg.tile_rows;
    if (cfg.test_stall) return;  // test hook: nothing issued, nothing in flight
    int cur = -1;
    const uint64_t run_len = cfg.tile_run > 1 ? (uint64_t)cfg.tile_run : 1ull;
    int64_t run = (int64_t)atomicAdd((unsigned long long*)tile_counter, run_len);
    uint64_t taken = 0;
    // the stage index and its barrier phase advance with each tile (a 64-bit
    // division by the run-time stage count per tile costs more than the tile's
    // own bookkeeping)
    for (int s = 0, parity = 0;; s = s + 1 == NS ? 0 : s + 1, parity ^= s == 0) {
        if (!mbar_wait(&empty[s], (uint32_t)parity ^ 1u, (uint32_t)cfg.wait_polls)) {
            set_error(descs[0].ctrl, kErrTimeout);
            return;
        }
        const int64_t t = run + (int64_t)taken;
        StageHdr& h = hdr[s];
        if (t >= cfg.total_tiles) {
            h.tile = -1;
            mbar_arrive(&full[s]);
            return;
        }
        if (++taken == run_len) {  // the run is used up: fetch the next one now
            run = (int64_t)atomicAdd((unsigned long long*)tile_counter, run_len);
            taken = 0;
        }
        int inst = cur < 0 ? 0 : cur;
        if (cfg.num_desc > 1)
            while (inst + 1 < cfg.num_desc && descs[inst + 1].tile_begin <= t) ++inst;
        if (inst != cur) {
            const uint64_t* src = reinterpret_cast<const uint64_t*>(&descs[inst]);
            uint64_t* dst = reinterpret_cast<uint64_t*>(pd);
            for (int i = 0; i < (int)(sizeof(BatchDesc) / 8); ++i) dst[i] = src[i];
            cur = inst;
        }
        const BatchDesc& d = *pd;
        int64_t row0 = (t - d.tile_begin) * (int64_t)T;
        int64_t left = d.num_rows - row0;
        int rows = (int)(left < T ? left : T);
        h.tile = t;
        h.row0 = row0;
        h.inst = inst;
        h.rows = rows;
        unsigned char* st = stage0 + (size_t)s * cfg.lay.stage_bytes;
        bool bulk = d.tma && rows == T;
        h.staged = bulk ? 1 : 0;
        uint32_t bytes = 0;
        for (int c = 0; c < P.num_cols; ++c) {
            int w = P.col_width[c];
            uint32_t db = w ? (uint32_t)(T * w) : (uint32_t)(T / 8);
            const char* src = d.col_data[c] + (w ? row0 * w : row0 / 8);
            h.view.data[c] = bulk ? (const char*)(st + cfg.lay.data_off[c]) : src;
            bytes += bulk ? db : 0;
            h.view.remap[c] = d.col_remap[c];
            h.view.remap_n[c] = d.col_remap_n[c];
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

// One op over a hash-tier chunk: raw row values -> global representation ->
// (optional) combine over key peers in the warp -> atomics on the row's slot
// (shared cache or HBM). Kind K is a compile-time constant.
template <int K, int R>
VR_DEV void hash_op(const OpDesc& op, const TileView& v, const int64_t (&r)[R], const bool (&live)[R],
                    uint64_t* const (&slot)[R], const bool (&in_smem)[R], const PeerPlan (&pp)[R], bool warp_agg) {
    OpDesc o;
    OpView ov;
    make_opview(op, v, o, ov);
#pragma unroll
    for (int j = 0; j < R; ++j) {
        Contrib c;
        if (live[j])
            op_raw<K>(o, ov, r[j], c);
        else
            czero(c);
        raw_to_global<K>(o, c);
        if (warp_agg) peer_reduce<K>(o, pp[j], c);
        if (slot[j]) {
            if (in_smem[j])
                apply_global<K, true>(o, slot[j] + o.word, c);
            else
                apply_global<K, false>(o, slot[j] + o.word, c);
        }
    }
}

// a * b * c in int64 (c = 1 for two factors); `fits` false when a product
// leaves int64. Out of line, so the per-row fast path stays one short branch
// (measured: 0.709 against 0.726 ms per 60M decimal-report rows).
static __noinline__ __device__ int64_t product_int64(int64_t a, int64_t b, int64_t c, bool& fits) {
    const int64_t p = a * b;
    fits = __mul64hi(a, b) == (p >> 63);
    const int64_t q = p * c;
    fits = fits && __mul64hi(p, c) == (q >> 63);
    return q;
}

// Kinds whose thread-private update is one int64 add per row.
template <int K>
struct OneAdd {
    static constexpr bool value =
        K == OP_COUNT_ROWS || K == OP_COUNT_VALID || K == OP_SUM_I32 || K == OP_SUM_I64 || K == OP_SUM_PROD;
};

// A OneAdd kind's value for row r without branches. `exact` false sends the
// row to the exact path instead (a null product factor, a product past int64
// or past its precision); the value is then 0.
template <int K, class V>
VR_DEV int64_t fast_value(const OpDesc& o, const V& v, int64_t r, bool& exact) {
    exact = true;
    switch (K) {
        case OP_COUNT_ROWS:
            return 1;
        case OP_COUNT_VALID:
            return (o.nterms > 0 ? terms_valid(o, v, r) : in_valid(o, v, o.col, r)) ? 1 : 0;
        case OP_SUM_I32:
            return in_valid(o, v, o.col, r) ? (int64_t)ld_i32(v, o.col, r) : 0;
        case OP_SUM_I64:
            return in_valid(o, v, o.col, r) ? ld_int(v, o.col, o.lane, r) : 0;
        case OP_SUM_PROD: {
            const int64_t a = term_value(o, v, r, 0), b = term_value(o, v, r, 1);
            const int64_t c = o.nterms == 3 ? term_value(o, v, r, 2) : 1;
            // factors within 32 bits (decimal(9, s) terms, and the values of
            // most wider ones): widening 32-bit multiplies, exact in int64 when
            // a three-factor product's first product also fits 32 bits. The
            // whole warp takes one path (direct-tier chunks keep every lane).
            const int64_t ab32 = (int64_t)(int32_t)a * (int32_t)b;
            const bool small =
                a == (int32_t)a && b == (int32_t)b && c == (int32_t)c && (o.nterms != 3 || ab32 == (int32_t)ab32);
            int64_t p;
            bool fits;
            if (__all_sync(kFull, small)) {
                p = o.nterms == 3 ? (int64_t)(int32_t)ab32 * (int32_t)c : ab32;
                fits = true;
            } else {
                p = product_int64(a, b, c, fits);
            }
            exact = fits && within_precision64(p, o.prec) && terms_valid(o, v, r);
            return exact ? p : 0;
        }
    }
    return 0;
}

// One op over a direct-tier chunk: thread-private hot words, CTA cold words.
// Rows that must not count (past the tile, unselected, a key outside its
// dictionary) arrive with the trash group, so the fast path has no branch per
// row: one int64 add into the row's hot word, its signed wrap and any need
// for the exact path noted in bit masks, handled after the chunk (rare).
// `pre` / `pre_op`: the chunk's products of the last two-factor product op
// (index pre_op, -1: none) that took the 32-bit path, for a three-factor op
// that extends it by one factor (OpDesc::prefix_op).
template <int K, int R, bool SM>
VR_DEV void direct_op(const OpDesc& op, const TileView& v, const int64_t (&r)[R], const int (&g)[R], uint64_t* priv,
                      uint64_t* cold, int nt, int ctid, int hw, int aw, int opi, int64_t (&pre)[R], int& pre_op) {
    OpDesc o;
    OpViewT<SM> ov;
    make_opview(op, v, o, ov);
    uint64_t* hot = priv + (size_t)o.hword * nt + ctid;
    uint64_t* cop = cold + o.word;
    const size_t gstride = (size_t)hw * nt;
    if constexpr (K == OP_SUM_PROD) {
        // The chunk's products when every factor of the warp's R rows fits 32
        // bits (one vote for the chunk): widening multiplies, and no per-row
        // exactness bookkeeping (measured: 0.650 against 0.674 ms per 60M
        // decimal-report rows). Otherwise the per-row path below.
        int64_t p[R];
        bool small = true;
        if (o.nterms == 3 && o.prefix_op > 0 && pre_op == o.prefix_op - 1) {
            // the first two factors' product: the earlier op's, this chunk
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const int64_t c = term_value(o, ov, r[j], 2);
                small = small && pre[j] == (int32_t)pre[j] && c == (int32_t)c;
                p[j] = (int64_t)(int32_t)pre[j] * (int32_t)c;
                small = small && within_precision64(p[j], o.prec) && terms_valid(o, ov, r[j]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const int64_t a = term_value(o, ov, r[j], 0), b = term_value(o, ov, r[j], 1);
                const int64_t c = o.nterms == 3 ? term_value(o, ov, r[j], 2) : 1;
                const int64_t ab32 = (int64_t)(int32_t)a * (int32_t)b;
                small = small && a == (int32_t)a && b == (int32_t)b && c == (int32_t)c &&
                        (o.nterms != 3 || ab32 == (int32_t)ab32);
                p[j] = o.nterms == 3 ? (int64_t)(int32_t)ab32 * (int32_t)c : ab32;
                small = small && within_precision64(p[j], o.prec) && terms_valid(o, ov, r[j]);
            }
        }
        if (__all_sync(kFull, small)) {
            if (o.nterms == 2) {
#pragma unroll
                for (int j = 0; j < R; ++j) pre[j] = p[j];
                pre_op = opi;
            }
            uint32_t wrap = 0;
#pragma unroll
            for (int j = 0; j < R; ++j) {
                uint64_t* h = hot + g[j] * gstride;
                const int64_t s = (int64_t)*h;
                const int64_t ns = (int64_t)((uint64_t)s + (uint64_t)p[j]);
                *h = (uint64_t)ns;
                wrap |= (uint32_t)(((s ^ ns) & (p[j] ^ ns)) < 0) << j;
            }
            if (wrap) {
#pragma unroll
                for (int j = 0; j < R; ++j)
                    if ((wrap >> j) & 1u)  // +-2^64 into the carry-save high word (+-2^32 there)
                        s_add(cop + (size_t)g[j] * aw + 1, p[j] > 0 ? (1ull << 32) : (0ull - (1ull << 32)));
            }
            return;
        }
    }
    if constexpr (OneAdd<K>::value) {
        constexpr bool kWraps = K == OP_SUM_I64 || K == OP_SUM_PROD;
        uint32_t rare = 0, wrap = 0;
        int64_t x[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            bool exact;
            x[j] = fast_value<K>(o, ov, r[j], exact);
            uint64_t* h = hot + g[j] * gstride;
            const int64_t s = (int64_t)*h;
            const int64_t ns = (int64_t)((uint64_t)s + (uint64_t)x[j]);
            *h = (uint64_t)ns;
            if (kWraps) wrap |= (uint32_t)(((s ^ ns) & (x[j] ^ ns)) < 0) << j;
            rare |= (uint32_t)!exact << j;
        }
        if (rare | wrap) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                if ((wrap >> j) & 1u)  // +-2^64 into the carry-save high word (+-2^32 there)
                    s_add(cop + (size_t)g[j] * aw + 1, x[j] > 0 ? (1ull << 32) : (0ull - (1ull << 32)));
                if ((rare >> j) & 1u) {
                    Contrib c;
                    if (op_raw<K>(o, ov, r[j], c)) apply_private<K>(o, hot + g[j] * gstride, nt, cop + (size_t)g[j] * aw, c);
                }
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            Contrib c;
            if (op_raw<K>(o, ov, r[j], c)) apply_private<K>(o, hot + g[j] * gstride, nt, cop + (size_t)g[j] * aw, c);
        }
    }
}

#ifdef VR_JIT
// Defined by the per-spec source after this header: jit_for_op(i, f) calls
// f(op, KindTag<kind>{}) with op i's descriptor as a compile-time constant;
// the key fields likewise. VR_JIT_NUM_OPS is the spec's op count.
template <class F>
VR_DEV void jit_for_op(int i, F&& f);
template <bool SM>
VR_DEV int jit_direct_index(const TileView& v, int64_t r);
template <int KW>
VR_DEV void jit_pack_key(const TileView& v, int64_t r, uint64_t (&k)[KW], bool& side, bool& bad);
#define VR_NUM_OPS(P) VR_JIT_NUM_OPS
#else
#define VR_NUM_OPS(P) ((P).num_ops)
#endif

// Launch and layout constants: compile-time in a per-spec kernel (so the
// compiler sees, e.g., that two ops' accumulator words never alias), read
// from the Program / launch config in the prebuilt one.
#ifdef VR_JIT
#define VR_THREADS(cfg) VR_JIT_THREADS
#define VR_PKW(P) VR_JIT_KW
#define VR_PHW(P) VR_JIT_HW
#define VR_PAW(P) VR_JIT_AW
#define VR_PSW(P) VR_JIT_SW
#define VR_PDSLOTS(P) ((int64_t)VR_JIT_DSLOTS)
#else
#define VR_THREADS(cfg) ((cfg).consumer_threads)
#define VR_PKW(P) ((P).kw)
#define VR_PHW(P) ((P).hw)
#define VR_PAW(P) ((P).aw)
#define VR_PSW(P) ((P).sw)
#define VR_PDSLOTS(P) ((P).direct_slots)
#endif

// f(op, KindTag<op kind>{}) for op i: the per-spec constant descriptor under
// VR_JIT, else the program's descriptor with its kind dispatched at run time.
template <class F>
VR_DEV void for_op(const Program& P, int i, F&& f) {
#ifdef VR_JIT
    (void)P;
    jit_for_op(i, f);
#else
    const OpDesc& op = P.ops[i];
    dispatch_kind(op.kind, [&](auto tag) { f(op, tag); });
#endif
}

// Hash tier: a chunk of R rows per consumer thread (row r[j]; warps stay
// converged: every lane runs every j). Each row's key is resolved to a slot
// (shared cache first, then HBM, else deferred); then every op runs once over
// the chunk with its kind fixed at compile time, so the per-row work is
// straight-line code.
template <int KW, int R>
VR_DEV void hash_chunk(const Program& P, const BatchDesc& D, const TileView& v, const int64_t (&r)[R],
                       const bool (&live_in)[R], int64_t row_base, uint64_t* scache, int sslots, int s_probes,
                       int g_probes, bool warp_agg, uint32_t& new_groups) {
    const int lane = threadIdx.x & 31;
    bool live[R];
    uint64_t* slot[R];
    bool in_smem[R];
    PeerPlan pp[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        live[j] = live_in[j];
        uint64_t key[KW];
        bool side = false;
        uint64_t h = 0;
        if (live[j]) {
            bool bad;
#ifdef VR_JIT
            jit_pack_key<KW>(v, r[j], key, side, bad);
#else
            pack_key<KW>(P, v, r[j], key, side, bad);
#endif
            if (bad) {
                set_error(D.ctrl, kErrBadKey);
                live[j] = false;
            }
            h = hash_key<KW>(key);
        }
        if (!live[j]) {
#pragma unroll
            for (int i = 0; i < KW; ++i) key[i] = 0;
        }
        uint32_t peers = 1u << lane;
        bool leader = live[j];
        pp[j].steps = 0;
        pp[j].recv = 0;
        if (warp_agg) {
            uint32_t livemask = __ballot_sync(kFull, live[j]);
            uint32_t m = kFull;
#pragma unroll
            for (int i = 0; i < KW; ++i) m &= __match_any_sync(kFull, (unsigned long long)key[i]);
            m &= live[j] ? livemask : ~livemask;
            peers = m;
            leader = live[j] && ((__ffs(peers) - 1) == lane);
            pp[j] = make_peer_plan(peers, lane);
        }
        slot[j] = nullptr;
        in_smem[j] = false;
        bool defer = false;
        if (leader) {
            bool fresh = false, to = false;
            if (sslots > 0 && !side) {
                slot[j] = find_or_insert<true, KW>(scache, sslots - 1, VR_PSW(P), key, h >> 32, false, s_probes, fresh, to);
                in_smem[j] = slot[j] != nullptr;
            }
            if (!slot[j]) {
                slot[j] = find_or_insert<false, KW>(D.table, D.cap_mask, VR_PSW(P), key, h, side, g_probes, fresh, to);
                if (slot[j] && fresh) ++new_groups;
                if (to) set_error(D.ctrl, kErrLockTimeout);
                defer = (slot[j] == nullptr) && !to;
            }
        }
        if (warp_agg) {
            uint32_t dm = __ballot_sync(kFull, defer);
            if (dm) defer = live[j] && ((dm >> (__ffs(peers) - 1)) & 1u);
        }
        if (defer) defer_row(D, row_base + r[j]);
        if (slot[j]) slot[j] += VR_PKW(P);  // accumulator words
    }
    VR_UNROLL
    for (int i = 0; i < VR_NUM_OPS(P); ++i)
        for_op(P, i, [&](const OpDesc& op, auto tag) {
            hash_op<decltype(tag)::value, R>(op, v, r, live, slot, in_smem, pp, warp_agg);
        });
}

// Direct tier: hot word h of group g of consumer thread t at
// priv[(g * hw + h) * nt + t]; the CTA's cold words of group g at
// cold[g * aw + word]. A chunk of R rows per thread, every op once per chunk
// (kind fixed at compile time, column pointers in registers).
template <int R, bool SM>
VR_DEV void direct_chunk(const Program& P, const BatchDesc& D, const TileView& v, const int64_t (&r)[R],
                         const bool (&live)[R], uint64_t* priv, uint64_t* cold, int nt, int ctid) {
    int g[R];
    uint32_t bad = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
#ifdef VR_JIT
        const int gi = jit_direct_index<SM>(v, r[j]);
        const bool ok = (unsigned)gi < (unsigned)VR_PDSLOTS(P);
#else
        const int64_t gi = direct_index(P, v, r[j]);
        const bool ok = gi >= 0 && gi < VR_PDSLOTS(P);
#endif
        bad |= (uint32_t)(live[j] && !ok) << j;
        // rows that do not count accumulate into the trash group (never flushed)
        g[j] = live[j] && ok ? (int)gi : (int)VR_PDSLOTS(P);
    }
    if (bad) set_error(D.ctrl, kErrBadKey);
    const int hw = VR_PHW(P), aw = VR_PAW(P);
    int64_t pre[R];
    int pre_op = -1;
    VR_UNROLL
    for (int i = 0; i < VR_NUM_OPS(P); ++i)
        for_op(P, i, [&](const OpDesc& op, auto tag) {
            direct_op<decltype(tag)::value, R, SM>(op, v, r, g, priv, cold, nt, ctid, hw, aw, i, pre, pre_op);
        });
}

// Direct tier flush: each consumer thread takes whole (group, op) pairs,
// combines the op's hot words over all consumer threads, adds the CTA's cold
// words, and applies both to the dense HBM table with atomics.
VR_DEV void flush_direct(const Program& P, const BatchDesc& D, uint64_t* priv, uint64_t* cold, int nt, int ctid) {
    const int64_t G = VR_PDSLOTS(P);
    const int nops = P.num_ops;
    #pragma unroll 1  // once per CTA: keep it small
    for (int64_t q = ctid; q < G * nops; q += nt) {
        int64_t g = q / nops;
        uint64_t* gslot = D.table + (size_t)g * VR_PSW(P);
        Contrib c;
        bool rows_op = false;
        for_op(P, (int)(q % nops), [&](const OpDesc& o, auto tag) {
            constexpr int K = decltype(tag)::value;
            private_to_global<K>(o, priv + ((size_t)g * VR_PHW(P) + o.hword) * nt, nt, c);
            apply_global<K, false>(o, gslot + VR_PKW(P) + o.word, c);
            Contrib cc;
            load_state(o, cold + (size_t)g * VR_PAW(P) + o.word, cc);
            apply_global<K, false>(o, gslot + VR_PKW(P) + o.word, cc);
            rows_op = K == OP_COUNT_ROWS;
        });
        if (rows_op && c.a != 0) {  // the group exists: store its key (same bits from every CTA)
            uint64_t kbuf[kMaxKW];
            direct_key(P, g, kbuf);
            for (int i = 0; i < VR_PKW(P); ++i) gslot[i] = kbuf[i];
        }
    }
}

// Is slot occupied? Every live group has COUNT_ROWS (word 0) >= 1.
VR_DEV bool slot_used(const Program& P, const uint64_t* slot) { return slot[VR_PKW(P)] != 0; }

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
    uint64_t* slot = find_or_insert<false, KW>(D.table, D.cap_mask, VR_PSW(P), key, hash_key<KW>(key), side, g_probes,
                                               fresh, to);
    if (to) set_error(D.ctrl, kErrLockTimeout);
    if (!slot) return false;
    if (fresh) ++new_groups;
    VR_UNROLL
    for (int i = 0; i < VR_NUM_OPS(P); ++i)
        for_op(P, i, [&](const OpDesc& o, auto tag) {
            Contrib c;
            load_state(o, src + KW + o.word, c);
            apply_global<decltype(tag)::value, false>(o, slot + KW + o.word, c);
        });
    return true;
}

// Hash tier flush: every occupied shared slot into HBM; slots HBM cannot
// take go to the spill list (merged by the host after the table grows).
template <int KW>
VR_DEV void flush_hash(const Program& P, const BatchDesc& D, uint64_t* scache, int sslots, int nt, int ctid,
                       uint32_t& new_groups, int g_probes) {
    #pragma unroll 1  // once per CTA: keep it small
    for (int i = ctid; i < sslots; i += nt) {
        const uint64_t* s = scache + (size_t)i * VR_PSW(P);
        if (!slot_used(P, s)) continue;
        if (!merge_state<KW>(P, D, s, new_groups, g_probes)) {
            unsigned long long k = atomicAdd((unsigned long long*)&D.ctrl[CTRL_SPILLED], 1ull);
            if ((int64_t)k < D.spill_cap) {
                uint64_t* dst = D.spill + (size_t)k * VR_PSW(P);
                for (int w = 0; w < VR_PSW(P); ++w) dst[w] = s[w];
            } else {
                set_error(D.ctrl, kErrSpillFull);
            }
        }
    }
}

VR_DEV void zero_words(uint64_t* p, int64_t n, int tid, int nt) {
    #pragma unroll 1  // once per CTA: keep it small
    for (int64_t i = tid; i < n; i += nt) p[i] = 0;
}

// Direct tier: one tile in chunks of R rows per consumer thread. SM: the
// tile's column data sits in the stage (shared-memory loads).
template <int R, bool SM>
VR_DEV void direct_tile(const Program& P, const BatchDesc& D, const TileView& v, int rows, uint64_t* tier, int NT,
                        int ctid) {
    for (int base = 0; base < rows; base += R * NT) {
        int64_t r[R];
        bool live[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int rr = base + j * NT + ctid;
            live[j] = rr < rows && (v.sel == nullptr || bit_at(v.sel, rr));
            r[j] = rr < rows ? rr : rows - 1;  // past the tile: a real row, counted into the trash group
        }
        direct_chunk<R, SM>(P, D, v, r, live, tier, tier + (size_t)(VR_PDSLOTS(P) + 1) * VR_PHW(P) * NT, NT, ctid);
    }
}

// One staged tile of `rows` rows, in chunks of R rows per consumer thread
// (row base + j * NT + ctid for j < R). The host sizes direct-tier tiles to
// exactly NT * R rows, so a full tile is one chunk with every lane busy.
// `staged`: the producer bulk-copied the tile's column data into the stage
// (every full tile of a 16-byte aligned batch); otherwise the view points
// at the batch's own buffers.
template <int KW, int TIER, int R>
VR_DEV void consume_tile(const Program& P, const BatchDesc& D, const LaunchCfg& cfg, const TileView& view, int rows,
                         bool staged, int64_t row0, uint64_t* tier, int sslots, int NT, int ctid,
                         uint32_t& new_groups) {
#ifdef VR_JIT
    // A register copy of the tile's column pointers: the per-spec kernel
    // names every column by a constant, so only the ones it reads stay live,
    // and stores to the accumulators cannot force them to be re-read.
    const TileView v = view;
#else
    const TileView& v = view;
#endif
    if (TIER == kTierDirect) {
#ifdef VR_JIT
        if (staged)
            direct_tile<R, true>(P, D, v, rows, tier, NT, ctid);
        else
            direct_tile<R, false>(P, D, v, rows, tier, NT, ctid);
#else
        (void)staged;
        direct_tile<R, false>(P, D, v, rows, tier, NT, ctid);
#endif
    } else {
        const int ss = D.smem_slots < sslots ? D.smem_slots : sslots;
#if defined(VR_JIT) && !VR_JIT_WARP_AGG
        // compiled for launches that never pre-aggregate in the warp: the
        // __match_any_sync and peer-reduction code folds away
        constexpr bool wa = false;
#else
        const bool wa = D.warp_agg != 0;
#endif
        for (int base = 0; base < rows; base += R * NT) {  // uniform trip count: warps stay converged
            int64_t r[R];
            bool live[R];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                r[j] = base + j * NT + ctid;
                live[j] = r[j] < rows && (v.sel == nullptr || bit_at(v.sel, r[j]));
            }
            hash_chunk<KW, R>(P, D, v, r, live, row0, tier, ss, D.s_probes, cfg.g_probes, wa, new_groups);
        }
    }
}

// ---------------------------------------------------------- the kernel ---
// The kernel body; the ahead-of-time kernel (agg_kernels.cu) and the per-spec
// kernels compiled at run time (jit.cpp) both wrap it.
template <int KW, int TIER>
VR_DEV void aggregate_body(const BatchDesc* __restrict__ descs, const LaunchCfg& cfg, uint64_t* __restrict__ tile_counter,
                           unsigned char* smem) {
    const SmemMap m = smem_map_impl(cfg.stages, cfg.lay.stage_bytes, cfg.tier_bytes);
    const Program& P = VR_PROG(smem + m.prog);
    BatchDesc& D = *reinterpret_cast<BatchDesc*>(smem + m.desc);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + m.bars);
    uint64_t* empty = full + kMaxStages;
    StageHdr* hdr = reinterpret_cast<StageHdr*>(smem + m.hdr);
    unsigned char* stage0 = smem + m.stages;
    uint64_t* tier = reinterpret_cast<uint64_t*>(smem + m.tier);

    const int tid = threadIdx.x;
    const int NT = VR_THREADS(cfg);
#ifndef VR_JIT
    coop_copy(smem + m.prog, descs[0].prog, (int)sizeof(Program), tid, blockDim.x);
#endif
    if (tid == 0) {
        for (int s = 0; s < cfg.stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], (uint32_t)(NT / 32));
        }
    }
    __syncthreads();

    if (tid >= NT) {  // producer warp
        if (tid == NT)
            producer_loop(P, descs, cfg, tile_counter, full, empty, hdr, stage0,
                          reinterpret_cast<BatchDesc*>(smem + m.pdesc));
        return;
    }

    // consumer warps
    const int ctid = tid;
    const int sslots = cfg.tier_bytes / (8 * VR_PSW(P));
    int cur = -1;
    uint32_t new_groups = 0;
    const int NS = cfg.stages;
    for (int s = 0, parity = 0;; s = s + 1 == NS ? 0 : s + 1, parity ^= s == 0) {
        if (!mbar_wait(&full[s], (uint32_t)parity, (uint32_t)cfg.wait_polls)) {
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
                    flush_direct(P, D, tier, tier + (size_t)(VR_PDSLOTS(P) + 1) * VR_PHW(P) * NT, NT, ctid);
                } else {
                    flush_hash<KW>(P, D, tier, D.smem_slots < sslots ? D.smem_slots : sslots, NT, ctid, new_groups,
                                   cfg.g_probes);
                }
                if (new_groups) atomicAdd((unsigned long long*)&D.ctrl[CTRL_GROUPS], (unsigned long long)new_groups);
                new_groups = 0;
                consumer_bar(NT);
            }
            coop_copy(&D, &descs[inst], (int)sizeof(BatchDesc), ctid, NT);
            // the next instance's part of the tier area (a batched launch
            // mixes small whole tables and hot-key caches)
            const int used = TIER == kTierDirect ? cfg.tier_bytes / 8
                                                 : min(descs[inst].smem_slots, sslots) * VR_PSW(P);
            zero_words(tier, used, ctid, NT);
            consumer_bar(NT);
            cur = inst;
        }
        const TileView& v = h.view;
#ifdef VR_JIT
        consume_tile<KW, TIER, VR_JIT_RCHUNK>(P, D, cfg, v, h.rows, h.staged != 0, h.row0, tier, sslots, NT, ctid,
                                                       new_groups);
#else
        // uniform: the host picks 2, 4 or 8 for direct-tier tiles, 1 for the hash tier
        if (TIER != kTierDirect)
            consume_tile<KW, TIER, 1>(P, D, cfg, v, h.rows, h.staged != 0, h.row0, tier, sslots, NT, ctid,
                                                       new_groups);
        else if (cfg.rchunk == 8)
            consume_tile<KW, TIER, 8>(P, D, cfg, v, h.rows, h.staged != 0, h.row0, tier, sslots, NT, ctid,
                                                       new_groups);
        else if (cfg.rchunk == 2)
            consume_tile<KW, TIER, 2>(P, D, cfg, v, h.rows, h.staged != 0, h.row0, tier, sslots, NT, ctid,
                                                       new_groups);
        else
            consume_tile<KW, TIER, 4>(P, D, cfg, v, h.rows, h.staged != 0, h.row0, tier, sslots, NT, ctid,
                                                       new_groups);
#endif
        __syncwarp();
        if ((ctid & 31) == 0) mbar_arrive(&empty[s]);
    }
    if (cur >= 0) {
        consumer_bar(NT);
        if (TIER == kTierDirect) {
            flush_direct(P, D, tier, tier + (size_t)(VR_PDSLOTS(P) + 1) * VR_PHW(P) * NT, NT, ctid);
        } else {
            flush_hash<KW>(P, D, tier, D.smem_slots < sslots ? D.smem_slots : sslots, NT, ctid, new_groups,
                           cfg.g_probes);
        }
        if (new_groups) atomicAdd((unsigned long long*)&D.ctrl[CTRL_GROUPS], (unsigned long long)new_groups);
    }
}

}  // namespace vr
