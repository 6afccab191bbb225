// Device building blocks of the grouped aggregate: PTX wrappers for the
// bulk-copy pipeline (mbarrier + cp.async.bulk), shared/global atomics,
// order-preserving keys, key packing, table probes and the per-op row
// contribution / accumulator apply logic.
//
// Semantics follow the reference's accumulators
// (kernels/src/main/java/io/vecruntime/kernels/GroupedAccumulators.java):
//   Count          :1010-1200  -> OP_COUNT_ROWS / OP_COUNT_VALID
//   LongSum        :363-624    -> OP_SUM_I32 / OP_SUM_I64 (exact carry-save; wrap or
//                                 ANSI check decided on the exact total at emit)
//   DoubleSum      :195-334    -> OP_SUM_F64 (compensated atomics)
//   WideLongSum    :637-1007   -> OP_SUM_I64 / OP_SUM_D128 (exact, order independent)
//   LongMinMax / DoubleMinMax / Decimal128MinMax :1203-1462 -> OP_MAX_KEY / OP_MAX_D128
// with Spark's NaN ordering (CompareOp.java:68-81, AggKernels.java:40-41).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vr_internal.h"

namespace vr {

#define VR_DEV __device__ __forceinline__

constexpr uint32_t kFull = 0xffffffffu;
// Spin limits: every wait in these kernels gives up after this many polls and
// reports kErrTimeout / kErrLockTimeout instead of hanging the device.
constexpr uint32_t kWaitPolls = 1u << 24;
constexpr uint32_t kLockPolls = 1u << 22;
// Single 64-bit keys are stored xor this constant so that 0 means "empty";
// the one key equal to it lives in an extra slot past the table's end.
constexpr uint64_t kSentinel = 0x9e3779b97f4a7c15ull;

// ---------------------------------------------------------------- PTX ----
VR_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

VR_DEV void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
VR_DEV void mbar_arrive(uint64_t* bar) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
        : "memory");
}
VR_DEV void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}
VR_DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false when the poll budget ran out.
VR_DEV bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitPolls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// One bulk copy global -> this CTA's shared memory, completing on `bar`.
// Both addresses 16-byte aligned, bytes a multiple of 16 (checked by the host).
VR_DEV void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// ----------------------------------------------------------- atomics ----
VR_DEV void s_add(uint64_t* p, uint64_t v) {
    asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(smem_u32(p)), "l"(v) : "memory");
}
VR_DEV void s_max(uint64_t* p, uint64_t v) {
    asm volatile("red.shared.max.u64 [%0], %1;" ::"r"(smem_u32(p)), "l"(v) : "memory");
}
VR_DEV void s_or(uint64_t* p, uint64_t v) {
    asm volatile("red.shared.or.b64 [%0], %1;" ::"r"(smem_u32(p)), "l"(v) : "memory");
}
VR_DEV double s_fadd(double* p, double v) {
    double old;
    asm volatile("atom.shared.add.f64 %0, [%1], %2;" : "=d"(old) : "r"(smem_u32(p)), "d"(v) : "memory");
    return old;
}
VR_DEV uint64_t s_cas(uint64_t* p, uint64_t cmp, uint64_t val) {
    uint64_t old;
    asm volatile("atom.shared.cas.b64 %0, [%1], %2, %3;"
                 : "=l"(old)
                 : "r"(smem_u32(p)), "l"(cmp), "l"(val)
                 : "memory");
    return old;
}
VR_DEV void g_add(uint64_t* p, uint64_t v) { atomicAdd((unsigned long long*)p, (unsigned long long)v); }
VR_DEV void g_max(uint64_t* p, uint64_t v) { atomicMax((unsigned long long*)p, (unsigned long long)v); }
VR_DEV void g_or(uint64_t* p, uint64_t v) { atomicOr((unsigned long long*)p, (unsigned long long)v); }
VR_DEV double g_fadd(double* p, double v) { return atomicAdd(p, v); }
VR_DEV uint64_t g_cas(uint64_t* p, uint64_t cmp, uint64_t val) {
    return (uint64_t)atomicCAS((unsigned long long*)p, (unsigned long long)cmp, (unsigned long long)val);
}
VR_DEV uint64_t ld_acquire_g(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
VR_DEV void st_release_g(uint64_t* p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
VR_DEV uint64_t ld_acquire_s(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.cta.shared.u64 %0, [%1];" : "=l"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}
VR_DEV void st_release_s(uint64_t* p, uint64_t v) {
    asm volatile("st.release.cta.shared.u64 [%0], %1;" ::"r"(smem_u32(p)), "l"(v) : "memory");
}
// 128-bit compare-and-swap (sm_90+): on failure (clo, chi) receive the value found.
VR_DEV bool g_cas128(uint64_t* p, uint64_t& clo, uint64_t& chi, uint64_t nlo, uint64_t nhi) {
    uint64_t olo, ohi;
    asm volatile(
        "{\n\t.reg .b128 d, c, s;\n\t"
        "mov.b128 c, {%2, %3};\n\t"
        "mov.b128 s, {%4, %5};\n\t"
        "atom.global.cas.b128 d, [%6], c, s;\n\t"
        "mov.b128 {%0, %1}, d;\n\t}"
        : "=l"(olo), "=l"(ohi)
        : "l"(clo), "l"(chi), "l"(nlo), "l"(nhi), "l"(p)
        : "memory");
    bool ok = (olo == clo && ohi == chi);
    clo = olo;
    chi = ohi;
    return ok;
}
VR_DEV bool s_cas128(uint64_t* p, uint64_t& clo, uint64_t& chi, uint64_t nlo, uint64_t nhi) {
    uint64_t olo, ohi;
    asm volatile(
        "{\n\t.reg .b128 d, c, s;\n\t"
        "mov.b128 c, {%2, %3};\n\t"
        "mov.b128 s, {%4, %5};\n\t"
        "atom.shared.cas.b128 d, [%6], c, s;\n\t"
        "mov.b128 {%0, %1}, d;\n\t}"
        : "=l"(olo), "=l"(ohi)
        : "l"(clo), "l"(chi), "l"(nlo), "l"(nhi), "r"(smem_u32(p))
        : "memory");
    bool ok = (olo == clo && ohi == chi);
    clo = olo;
    chi = ohi;
    return ok;
}
VR_DEV uint64_t ld_relaxed_g(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Address-space dispatch: S = true for shared memory, false for global.
template <bool S> struct Mem;
template <> struct Mem<true> {
    static VR_DEV void add(uint64_t* p, uint64_t v) { s_add(p, v); }
    static VR_DEV void max(uint64_t* p, uint64_t v) { s_max(p, v); }
    static VR_DEV void bor(uint64_t* p, uint64_t v) { s_or(p, v); }
    static VR_DEV double fadd(double* p, double v) { return s_fadd(p, v); }
    static VR_DEV uint64_t cas(uint64_t* p, uint64_t c, uint64_t v) { return s_cas(p, c, v); }
    static VR_DEV uint64_t ld_acq(const uint64_t* p) { return ld_acquire_s(p); }
    static VR_DEV void st_rel(uint64_t* p, uint64_t v) { st_release_s(p, v); }
    static VR_DEV uint64_t ld(const uint64_t* p) { return *(const volatile uint64_t*)p; }
    static VR_DEV bool cas128(uint64_t* p, uint64_t& clo, uint64_t& chi, uint64_t nlo, uint64_t nhi) {
        return s_cas128(p, clo, chi, nlo, nhi);
    }
};
template <> struct Mem<false> {
    static VR_DEV void add(uint64_t* p, uint64_t v) { g_add(p, v); }
    static VR_DEV void max(uint64_t* p, uint64_t v) { g_max(p, v); }
    static VR_DEV void bor(uint64_t* p, uint64_t v) { g_or(p, v); }
    static VR_DEV double fadd(double* p, double v) { return g_fadd(p, v); }
    static VR_DEV uint64_t cas(uint64_t* p, uint64_t c, uint64_t v) { return g_cas(p, c, v); }
    static VR_DEV uint64_t ld_acq(const uint64_t* p) { return ld_acquire_g(p); }
    static VR_DEV void st_rel(uint64_t* p, uint64_t v) { st_release_g(p, v); }
    static VR_DEV uint64_t ld(const uint64_t* p) { return ld_relaxed_g(p); }
    static VR_DEV bool cas128(uint64_t* p, uint64_t& clo, uint64_t& chi, uint64_t nlo, uint64_t nhi) {
        return g_cas128(p, clo, chi, nlo, nhi);
    }
};

// ----------------------------------------------------- ordered keys ----
// Order-preserving unsigned images: max over them is max over the values.
// Spark's NaN order: NaN (any payload, canonicalised) above +Inf; -0.0 below
// +0.0 as in Java's Math.min/max, which the reference's masked path uses.
VR_DEV uint64_t okey_i64(int64_t x) { return (uint64_t)x ^ 0x8000000000000000ull; }
VR_DEV int64_t okey_i64_dec(uint64_t k) { return (int64_t)(k ^ 0x8000000000000000ull); }
VR_DEV uint64_t okey_f64(double x) {
    uint64_t b = isnan(x) ? 0x7ff8000000000000ull : (uint64_t)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
VR_DEV double okey_f64_dec(uint64_t k) {
    uint64_t b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

// -------------------------------------------------------------- hash ----
VR_DEV uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
template <int KW> VR_DEV uint64_t hash_key(const uint64_t (&k)[KW]) {
    uint64_t h = 0x2545f4914f6cdd1dull;
#pragma unroll
    for (int i = 0; i < KW; ++i) h = mix64(h ^ k[i]);
    return h;
}

// --------------------------------------------------- 128-bit helpers ----
struct I128 {
    uint64_t lo;
    int64_t hi;
};
VR_DEV I128 mul_i64(int64_t a, int64_t b) {
    I128 r;
    r.lo = (uint64_t)a * (uint64_t)b;
    r.hi = __mul64hi(a, b);
    return r;
}
// Signed 128 x signed 64 -> 128, with overflow detection (false = overflow).
VR_DEV bool mul_i128_i64(I128 a, int64_t b, I128& out) {
    bool neg = (a.hi < 0) != (b < 0);
    // magnitudes
    uint64_t alo = a.lo, ahi = (uint64_t)a.hi;
    if (a.hi < 0) {
        alo = ~alo + 1;
        ahi = ~ahi + (alo == 0 ? 1 : 0);
    }
    uint64_t bm = b < 0 ? (uint64_t)0 - (uint64_t)b : (uint64_t)b;
    uint64_t p0lo = alo * bm, p0hi = __umul64hi(alo, bm);
    uint64_t p1lo = ahi * bm, p1hi = __umul64hi(ahi, bm);
    if (p1hi != 0) return false;
    uint64_t hi = p0hi + p1lo;
    if (hi < p0hi) return false;
    if (hi >> 63) {  // magnitude >= 2^127: only -2^127 representable
        if (!(neg && hi == 0x8000000000000000ull && p0lo == 0)) return false;
    }
    uint64_t lo = p0lo;
    if (neg) {
        lo = ~lo + 1;
        hi = ~hi + (lo == 0 ? 1 : 0);
    }
    out.lo = lo;
    out.hi = (int64_t)hi;
    return true;
}

// 10^p for p in [0, 38] as (lo, hi) words, uploaded once per device.
__constant__ uint64_t c_pow10_lo[39];
__constant__ uint64_t c_pow10_hi[39];

// |v| < 10^p for a signed 128-bit v (lo, hi).
VR_DEV bool within_precision(uint64_t lo, int64_t hi, int p) {
    uint64_t mlo = lo, mhi = (uint64_t)hi;
    if (hi < 0) {
        mlo = ~lo + 1;
        mhi = ~(uint64_t)hi + (mlo == 0 ? 1 : 0);
    }
    uint64_t plo = c_pow10_lo[p], phi = c_pow10_hi[p];
    return mhi < phi || (mhi == phi && mlo < plo);
}

// --------------------------------------------------------- columns ----
// A tile view: per staged column a base pointer (shared or global) with the
// tile's row 0 at index 0, and an optional validity bitmap with the same
// origin.
struct TileView {
    const char* data[kMaxCols];
    const uint32_t* valid[kMaxCols];
    const uint32_t* sel;
};

VR_DEV bool bit_at(const uint32_t* words, int64_t r) { return (words[r >> 5] >> (r & 31)) & 1u; }
VR_DEV bool col_valid(const TileView& v, int c, int64_t r) {
    const uint32_t* w = v.valid[c];
    return w == nullptr || bit_at(w, r);
}
VR_DEV int32_t ld_i32(const TileView& v, int c, int64_t r) {
    return reinterpret_cast<const int32_t*>(v.data[c])[r];
}
VR_DEV int64_t ld_i64(const TileView& v, int c, int64_t r) {
    return reinterpret_cast<const int64_t*>(v.data[c])[r];
}
VR_DEV uint64_t ld_u64(const TileView& v, int c, int64_t r) {
    return reinterpret_cast<const uint64_t*>(v.data[c])[r];
}
VR_DEV double ld_f64(const TileView& v, int c, int64_t r) {
    return reinterpret_cast<const double*>(v.data[c])[r];
}
VR_DEV I128 ld_d128(const TileView& v, int c, int64_t r) {
    const uint64_t* p = reinterpret_cast<const uint64_t*>(v.data[c]) + 2 * r;
    I128 x;
    x.lo = p[0];
    x.hi = (int64_t)p[1];
    return x;
}
// Integer lanes widened to int64 (INT32 / DICT32 sign-extended).
VR_DEV int64_t ld_int(const TileView& v, int c, int lane, int64_t r) {
    return lane == VR_INT32 || lane == VR_DICT32 ? (int64_t)ld_i32(v, c, r) : ld_i64(v, c, r);
}

// ------------------------------------------------------ key packing ----
// Packs row r's key tuple into KW words; `side` is set for the one single
// 64-bit key equal to kSentinel (sentinel layout only). Null keys store zero
// data and their null bit, as GroupKeyTable.insert does (GroupKeyTable.java:2515-2540).
template <int KW>
VR_DEV void pack_key(const Program& P, const TileView& v, int64_t r, uint64_t (&k)[KW], bool& side, bool& bad) {
#pragma unroll
    for (int i = 0; i < KW; ++i) k[i] = 0;
    side = false;
    bad = false;
    for (int f = 0; f < P.num_keys; ++f) {
        const KeyField& kf = P.keys[f];
        bool ok = col_valid(v, kf.col, r);
        if (!ok) {
            if (kf.null_word >= 0) k[kf.null_word] |= 1ull << kf.null_shift;
            continue;
        }
        switch (kf.lane) {
            case VR_INT32:
            case VR_DICT32: {
                uint32_t u = (uint32_t)ld_i32(v, kf.col, r);
                if (kf.bits < 32 && (u >> kf.bits) != 0) bad = true;  // id outside the declared dictionary
                k[kf.word] |= (uint64_t)u << kf.shift;
                break;
            }
            case VR_INT64:
            case VR_FLOAT64:
                k[kf.word] |= ld_u64(v, kf.col, r);
                break;
            case VR_BOOL:
                k[kf.word] |= (uint64_t)bit_at(reinterpret_cast<const uint32_t*>(v.data[kf.col]), r) << kf.shift;
                break;
            case VR_DECIMAL128: {
                I128 x = ld_d128(v, kf.col, r);
                k[kf.word] |= x.lo;
                if (kf.word + 1 < KW) k[kf.word + 1] |= (uint64_t)x.hi;
                break;
            }
        }
    }
    if (P.occ_word >= 0) {
        k[P.occ_word] |= 1ull << P.occ_shift;
    } else {  // sentinel layout: one 64-bit word, no spare bit
        side = (k[0] == kSentinel);
        k[0] ^= kSentinel;
    }
}

// Direct tier: the combination index of a row's dictionary / boolean keys;
// -1 when an id lies outside its declared dictionary.
VR_DEV int64_t direct_index(const Program& P, const TileView& v, int64_t r) {
    int64_t idx = 0;
    for (int f = 0; f < P.num_keys; ++f) {
        const KeyField& kf = P.keys[f];
        int64_t val;
        if (!col_valid(v, kf.col, r)) {
            val = kf.card - 1;  // null is the last value of a nullable field
        } else if (kf.lane == VR_BOOL) {
            val = bit_at(reinterpret_cast<const uint32_t*>(v.data[kf.col]), r);
        } else {
            val = (int64_t)(uint32_t)ld_i32(v, kf.col, r);
            if (val >= (int64_t)kf.card - (kf.null_word >= 0 ? 1 : 0)) return -1;  // id outside the dictionary
        }
        idx += val * kf.mul;
    }
    return idx;
}

// Direct tier: the packed key of a combination index (written at flush).
VR_DEV void direct_key(const Program& P, int64_t idx, uint64_t* out) {
    for (int i = 0; i < P.kw; ++i) out[i] = 0;
    for (int f = 0; f < P.num_keys; ++f) {
        const KeyField& kf = P.keys[f];
        int64_t val = (idx / kf.mul) % kf.card;
        bool is_null = kf.null_word >= 0 && val == kf.card - 1;
        if (is_null)
            out[kf.null_word] |= 1ull << kf.null_shift;
        else
            out[kf.word] |= (uint64_t)(uint32_t)val << kf.shift;
    }
    if (P.occ_word >= 0) out[P.occ_word] |= 1ull << P.occ_shift;
}

// ------------------------------------------------------ table probe ----
// Finds or inserts key k; returns the slot or nullptr when `max_probe` slots
// were full of other keys. `fresh` is set for the thread that inserted.
// Layouts:
//   sentinel (KW == 1, occ_word < 0): one CAS from 0; the key equal to the
//     sentinel uses the extra slot at index `cap` (caller passes side=true).
//   occupancy bit, KW == 1: one CAS from 0.
//   KW >= 2: claim the last word with a BUSY bit, write the other words,
//     then publish the last word (data | occupancy) with release semantics;
//     readers acquire the last word before comparing, so no torn key is ever
//     compared. Waits on a BUSY slot are bounded (kLockPolls).
template <bool S, int KW>
VR_DEV uint64_t* find_or_insert(uint64_t* table, int64_t mask, int sw, const uint64_t (&k)[KW], uint64_t h,
                                bool side, int max_probe, bool& fresh, bool& timeout) {
    fresh = false;
    if (side) {
        // the extra slot past the table: occupied by definition (emission tests its count)
        return table + (mask + 1) * (int64_t)sw;
    }
    int64_t pos = (int64_t)(h & (uint64_t)mask);
    for (int p = 0; p < max_probe; ++p) {
        uint64_t* slot = table + pos * (int64_t)sw;
        if (KW == 1) {
            uint64_t cur = Mem<S>::ld(slot);
            if (cur == k[0]) return slot;
            if (cur == 0) {
                uint64_t old = Mem<S>::cas(slot, 0, k[0]);
                if (old == 0) {
                    fresh = true;
                    return slot;
                }
                if (old == k[0]) return slot;
            }
        } else {
            constexpr uint64_t kBusy = 1ull << 62;
            uint64_t* last = slot + (KW - 1);
            uint64_t cur = Mem<S>::ld_acq(last);
            if (cur == 0) {
                uint64_t old = Mem<S>::cas(last, 0, kBusy);
                if (old == 0) {
#pragma unroll
                    for (int i = 0; i < KW - 1; ++i) slot[i] = k[i];
                    Mem<S>::st_rel(last, k[KW - 1]);
                    fresh = true;
                    return slot;
                }
                cur = old;
            }
            if (cur == kBusy) {
                uint32_t polls = 0;
                do {
                    cur = Mem<S>::ld_acq(last);
                } while (cur == kBusy && ++polls < kLockPolls);
                if (cur == kBusy) {
                    timeout = true;
                    return nullptr;
                }
            }
            if (cur == k[KW - 1]) {
                bool eq = true;
#pragma unroll
                for (int i = 0; i < KW - 1; ++i) eq &= (slot[i] == k[i]);
                if (eq) return slot;
            }
        }
        pos = (pos + 1) & mask;
    }
    return nullptr;
}

// ----------------------------------------------------- contributions ----
// One row's (or one warp's peers') contribution to an op: up to kMaxContrib
// words in the op's accumulator representation. All-zero == identity.
struct Contrib {
    uint64_t w[kMaxContrib];
};

// A row is "live" when it is inside the tile, selected and has a slot.
// Computes op `o`'s contribution of row r; returns false when the row adds
// nothing (invalid input), leaving c zeroed.
VR_DEV bool op_contrib(const OpDesc& o, const TileView& v, int64_t r, Contrib& c) {
#pragma unroll
    for (int i = 0; i < kMaxContrib; ++i) c.w[i] = 0;
    switch (o.kind) {
        case OP_COUNT_ROWS:
            c.w[0] = 1;
            return true;
        case OP_COUNT_VALID: {
            bool ok = true;
            if (o.nterms > 0) {
                for (int t = 0; t < o.nterms; ++t) ok &= col_valid(v, o.term_col[t], r);
            } else {
                ok = col_valid(v, o.col, r);
            }
            c.w[0] = ok ? 1 : 0;
            return ok;
        }
        case OP_SUM_I32: {
            if (!col_valid(v, o.col, r)) return false;
            c.w[0] = (uint64_t)(int64_t)ld_i32(v, o.col, r);
            return true;
        }
        case OP_SUM_I64: {
            if (!col_valid(v, o.col, r)) return false;
            int64_t x = ld_int(v, o.col, o.lane, r);
            c.w[0] = (uint64_t)(uint32_t)x;
            c.w[1] = (uint64_t)(int64_t)(int32_t)(x >> 32);
            return true;
        }
        case OP_SUM_F64: {
            if (!col_valid(v, o.col, r)) return false;
            double x = ld_f64(v, o.col, r);
            c.w[0] = (uint64_t)__double_as_longlong(x);
            c.w[1] = 0;  // +0.0
            return true;
        }
        case OP_SUM_D128: {
            if (!col_valid(v, o.col, r)) return false;
            I128 x = ld_d128(v, o.col, r);
            c.w[0] = (uint32_t)x.lo;
            c.w[1] = (uint32_t)(x.lo >> 32);
            c.w[2] = (uint32_t)(uint64_t)x.hi;
            c.w[3] = (uint64_t)(int64_t)(int32_t)(x.hi >> 32);
            return true;
        }
        case OP_SUM_PROD: {
            bool ok = true;
            for (int t = 0; t < o.nterms; ++t) ok &= col_valid(v, o.term_col[t], r);
            if (!ok) return false;
            // term values: addend + sign * column (INT64 unscaled lanes)
            int64_t t0 = o.term_add[0] + (o.term_sign[0] < 0 ? -ld_i64(v, o.term_col[0], r) : ld_i64(v, o.term_col[0], r));
            int64_t t1 = o.term_add[1] + (o.term_sign[1] < 0 ? -ld_i64(v, o.term_col[1], r) : ld_i64(v, o.term_col[1], r));
            I128 p = mul_i64(t0, t1);
            bool fits = true;
            if (o.nterms == 3) {
                int64_t t2 = o.term_add[2] +
                             (o.term_sign[2] < 0 ? -ld_i64(v, o.term_col[2], r) : ld_i64(v, o.term_col[2], r));
                I128 q;
                fits = mul_i128_i64(p, t2, q);
                p = q;
            }
            if (!fits || !within_precision(p.lo, p.hi, o.prec)) {
                // Spark's CheckOverflow on the product: null (non-ANSI) or an error (ANSI)
                if (o.flags & OPF_CHECKED) c.w[6] = 1;
                return (o.flags & OPF_CHECKED) != 0;
            }
            c.w[7] = 1;  // the row counts toward the sum (its product is not null)
            bool small = (p.hi == ((int64_t)p.lo >> 63));
            if (small) {
                int64_t x = (int64_t)p.lo;
                c.w[0] = (uint64_t)(uint32_t)x;
                c.w[1] = (uint64_t)(int64_t)(int32_t)(x >> 32);
            } else {
                c.w[2] = (uint32_t)p.lo;
                c.w[3] = (uint32_t)(p.lo >> 32);
                c.w[4] = (uint32_t)(uint64_t)p.hi;
                c.w[5] = (uint64_t)(int64_t)(int32_t)(p.hi >> 32);
            }
            return true;
        }
        case OP_MAX_KEY: {
            if (!col_valid(v, o.col, r)) return false;
            uint64_t k = o.lane == VR_FLOAT64 ? okey_f64(ld_f64(v, o.col, r)) : okey_i64(ld_int(v, o.col, o.lane, r));
            c.w[0] = (o.flags & OPF_MIN) ? ~k : k;
            return true;
        }
        case OP_MAX_D128: {
            if (!col_valid(v, o.col, r)) return false;
            I128 x = ld_d128(v, o.col, r);
            uint64_t lo = x.lo, hi = (uint64_t)x.hi ^ 0x8000000000000000ull;
            if (o.flags & OPF_MIN) {
                lo = ~lo;
                hi = ~hi;
            }
            c.w[0] = lo;
            c.w[1] = hi;
            return true;
        }
        case OP_MERGE_DSUM: {
            // WideDecimalSumMergeAgg.merge (VectorAggregates.scala:700-725): rows with a null or
            // true isEmpty are skipped; a null sum on a non-empty row poisons the group.
            const uint32_t* eb = reinterpret_cast<const uint32_t*>(v.data[o.col2]);
            bool empty_valid = col_valid(v, o.col2, r);
            if (!empty_valid || bit_at(eb, r)) return false;
            if (!col_valid(v, o.col, r)) {
                c.w[4] = kFlagNonEmpty | kFlagOverflow;
                return true;
            }
            I128 x = ld_d128(v, o.col, r);
            c.w[0] = (uint32_t)x.lo;
            c.w[1] = (uint32_t)(x.lo >> 32);
            c.w[2] = (uint32_t)(uint64_t)x.hi;
            c.w[3] = (uint64_t)(int64_t)(int32_t)(x.hi >> 32);
            c.w[4] = kFlagNonEmpty;
            return true;
        }
        case OP_MERGE_DAVG: {
            // WideDecimalAvgMergeAgg.merge (VectorAggregates.scala:557-573): counts add when valid;
            // a null sum poisons the group.
            bool any = false;
            if (col_valid(v, o.col2, r)) {
                int64_t n = ld_i64(v, o.col2, r);
                c.w[4] = (uint64_t)(uint32_t)n;
                c.w[5] = (uint64_t)(int64_t)(int32_t)(n >> 32);
                any = true;
            }
            if (!col_valid(v, o.col, r)) {
                c.w[6] = kFlagOverflow;
                return true;
            }
            I128 x = ld_d128(v, o.col, r);
            c.w[0] = (uint32_t)x.lo;
            c.w[1] = (uint32_t)(x.lo >> 32);
            c.w[2] = (uint32_t)(uint64_t)x.hi;
            c.w[3] = (uint64_t)(int64_t)(int32_t)(x.hi >> 32);
            (void)any;
            return true;
        }
    }
    return false;
}

// Kinds of an op's contribution words (mirrors the host's word_kind table).
VR_DEV uint8_t op_word_kind(const Program& P, const OpDesc& o, int i) { return P.word_kind[o.word + i]; }

// ------------------------------------------------- double-double add ----
VR_DEV void two_sum(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    if (!isfinite(s)) {
        e = 0.0;
        return;
    }
    double bb = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
VR_DEV void dd_add(double& s, double& c, double s2, double c2) {
    double t, e;
    two_sum(s, s2, t, e);
    s = t;
    c = __dadd_rn(c, __dadd_rn(c2, e));
}
VR_DEV bool u128_gt(uint64_t alo, uint64_t ahi, uint64_t blo, uint64_t bhi) {
    return ahi > bhi || (ahi == bhi && alo > blo);
}

// Combines contribution b into a (same op), word kind by word kind.
VR_DEV void contrib_combine(const Program& P, const OpDesc& o, Contrib& a, const Contrib& b) {
    for (int i = 0; i < o.nwords; ++i) {
        switch (op_word_kind(P, o, i)) {
            case WK_ADD: a.w[i] += b.w[i]; break;
            case WK_MAX: a.w[i] = a.w[i] > b.w[i] ? a.w[i] : b.w[i]; break;
            case WK_OR: a.w[i] |= b.w[i]; break;
            case WK_F64: {
                double s = __longlong_as_double((long long)a.w[i]), c = __longlong_as_double((long long)a.w[i + 1]);
                dd_add(s, c, __longlong_as_double((long long)b.w[i]), __longlong_as_double((long long)b.w[i + 1]));
                a.w[i] = (uint64_t)__double_as_longlong(s);
                a.w[i + 1] = (uint64_t)__double_as_longlong(c);
                ++i;
                break;
            }
            case WK_MAX128:
                if (u128_gt(b.w[i], b.w[i + 1], a.w[i], a.w[i + 1])) {
                    a.w[i] = b.w[i];
                    a.w[i + 1] = b.w[i + 1];
                }
                ++i;
                break;
            default: break;
        }
    }
}

// Applies a contribution to accumulator words `acc` (this op's first word)
// with atomics in shared (S) or global memory. Zero words are skipped: every
// word kind has identity 0.
template <bool S>
VR_DEV void contrib_apply(const Program& P, const OpDesc& o, uint64_t* acc, const Contrib& c) {
    for (int i = 0; i < o.nwords; ++i) {
        uint8_t kind = op_word_kind(P, o, i);
        switch (kind) {
            case WK_ADD:
                if (c.w[i]) Mem<S>::add(acc + i, c.w[i]);
                break;
            case WK_MAX:
                if (c.w[i]) Mem<S>::max(acc + i, c.w[i]);
                break;
            case WK_OR:
                if (c.w[i]) Mem<S>::bor(acc + i, c.w[i]);
                break;
            case WK_F64: {
                double s = __longlong_as_double((long long)c.w[i]);
                double cc = __longlong_as_double((long long)c.w[i + 1]);
                if (c.w[i] != 0 || c.w[i + 1] != 0) {
                    // Compensated atomic: the hardware add rounds to nearest like __dadd_rn,
                    // so the thread recovers the exact rounding error of its own add and
                    // accumulates it (and the incoming compensation) in the next word.
                    double old = Mem<S>::fadd(reinterpret_cast<double*>(acc + i), s);
                    double nw, err;
                    two_sum(old, s, nw, err);
                    double tot = __dadd_rn(err, cc);
                    if (tot != 0.0) Mem<S>::fadd(reinterpret_cast<double*>(acc + i + 1), tot);
                }
                ++i;
                break;
            }
            case WK_MAX128: {
                uint64_t lo = c.w[i], hi = c.w[i + 1];
                if (lo | hi) {
                    // 128-bit max by a 128-bit CAS loop (the pair is 16-byte aligned)
                    uint64_t clo = Mem<S>::ld(acc + i), chi = Mem<S>::ld(acc + i + 1);
                    for (int it = 0; it < 1 << 16 && u128_gt(lo, hi, clo, chi); ++it) {
                        if (Mem<S>::cas128(acc + i, clo, chi, lo, hi)) break;
                    }
                }
                ++i;
                break;
            }
            default: break;
        }
    }
}

// Thread-private (non-atomic) apply for the direct tier: word i of the op
// lives at acc[i * stride].
VR_DEV void contrib_apply_private(const Program& P, const OpDesc& o, uint64_t* acc, int stride, const Contrib& c) {
    for (int i = 0; i < o.nwords; ++i) {
        uint8_t kind = op_word_kind(P, o, i);
        uint64_t* p = acc + (int64_t)i * stride;
        switch (kind) {
            case WK_ADD:
                if (c.w[i]) *p += c.w[i];
                break;
            case WK_MAX:
                if (c.w[i] > *p) *p = c.w[i];
                break;
            case WK_OR:
                *p |= c.w[i];
                break;
            case WK_F64: {
                if (c.w[i] | c.w[i + 1]) {
                    uint64_t* q = acc + (int64_t)(i + 1) * stride;
                    double s = __longlong_as_double((long long)*p), cc = __longlong_as_double((long long)*q);
                    dd_add(s, cc, __longlong_as_double((long long)c.w[i]), __longlong_as_double((long long)c.w[i + 1]));
                    *p = (uint64_t)__double_as_longlong(s);
                    *q = (uint64_t)__double_as_longlong(cc);
                }
                ++i;
                break;
            }
            case WK_MAX128: {
                uint64_t* q = acc + (int64_t)(i + 1) * stride;
                if (u128_gt(c.w[i], c.w[i + 1], *p, *q)) {
                    *p = c.w[i];
                    *q = c.w[i + 1];
                }
                ++i;
                break;
            }
            default: break;
        }
    }
}

// ------------------------------------------------ warp peer reduction ----
// Peers are lanes holding the same key (from __match_any_sync). A tree over
// each peer group's ranks: at step s, the lane of rank r (r % 2^(s+1) == 0)
// takes the partial of rank r + 2^s. Rank -> lane uses nth_set_bit.
VR_DEV int nth_set_bit(uint32_t mask, int n) {
    // position of the n-th (0-based) set bit of mask; mask has > n set bits
    int pos = 0;
#pragma unroll
    for (int width = 16; width >= 1; width >>= 1) {
        uint32_t low = mask & ((1u << width) - 1u);
        int cnt = __popc(low);
        if (n >= cnt) {
            n -= cnt;
            mask >>= width;
            pos += width;
        } else {
            mask = low;
        }
    }
    return pos;
}

struct PeerPlan {
    int steps;
    int src[5];
    uint32_t recv;  // bit s: this lane receives at step s
};

VR_DEV PeerPlan make_peer_plan(uint32_t peers, int lane) {
    PeerPlan pp;
    int n = __popc(peers);
    int r = __popc(peers & ((1u << lane) - 1u));
    int maxn = (int)__reduce_max_sync(kFull, (unsigned)n);
    pp.steps = 0;
    while ((1 << pp.steps) < maxn) ++pp.steps;
    pp.recv = 0;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        pp.src[s] = lane;
        if (s < pp.steps) {
            int stride = 1 << s;
            if ((r % (2 * stride)) == 0 && r + stride < n) {
                pp.recv |= 1u << s;
                pp.src[s] = nth_set_bit(peers, r + stride);
            }
        }
    }
    return pp;
}

VR_DEV void peer_reduce(const Program& P, const OpDesc& o, const PeerPlan& pp, Contrib& c) {
    for (int s = 0; s < pp.steps; ++s) {
        Contrib t;
#pragma unroll
        for (int i = 0; i < kMaxContrib; ++i) {
            t.w[i] = (i < o.nwords) ? (uint64_t)__shfl_sync(kFull, (unsigned long long)c.w[i], pp.src[s]) : 0;
        }
        if (pp.recv & (1u << s)) contrib_combine(P, o, c, t);
    }
}

}  // namespace vr
