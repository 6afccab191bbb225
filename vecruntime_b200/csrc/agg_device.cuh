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
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>
#endif

#include "vr_internal.h"

namespace vr {

#define VR_DEV __device__ __forceinline__

// Per-spec compilation (NVRTC, jit.cpp) defines VR_JIT and a compile-time
// constant Program kJitProg: the program is then read from it (folded into
// the code) instead of from the shared-memory copy, and loops over ops and
// key fields unroll completely.
#ifdef VR_JIT
#define VR_PROG(smem_copy) (kJitProg)
#define VR_UNROLL _Pragma("unroll")
#else
#define VR_PROG(smem_copy) (*reinterpret_cast<const Program*>(smem_copy))
#define VR_UNROLL
#endif

constexpr uint32_t kFull = 0xffffffffu;
// Spin limits: every wait in these kernels gives up after this many polls and
// reports kErrTimeout / kErrLockTimeout instead of hanging the device.
constexpr uint32_t kSuspendHintNs = 1000000;  // at most 1 ms per poll
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
// try_wait with a suspend-time hint: the thread sleeps until the phase
// completes (or the hint, in ns, runs out) instead of spinning, so waiting
// warps leave the issue slots to the warps doing work.
VR_DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendHintNs)
        : "memory");
    return ok != 0;
}
// Bounded wait: false when the poll budget ran out (`polls` suspended polls
// of up to kSuspendHintNs each: about a second by default, never forever).
VR_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t polls) {
    for (uint32_t i = 0; i < polls; ++i)
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
// A 64-bit add to shared memory as two native 32-bit atomics: the low half
// returns its old value, from which the carry into the high half follows;
// the high half is touched only when its addend (with the carry) is not
// zero. Exact modulo 2^64 under any interleaving (each adder carries its own
// overflow). Measured on B200 shared memory: a 64-bit atomic add runs at 1.3
// per clock per SM (the hardware loops on a compare-and-swap), a 32-bit one
// at 9. Readers see a consistent word only after the adders are done (the
// tables are read after a barrier).
VR_DEV void s_add(uint64_t* p, uint64_t v) {
    const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
    const uint32_t a = smem_u32(p);
    uint32_t old;
    asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(a), "r"(lo) : "memory");
    const uint32_t h = hi + ((uint32_t)(old + lo) < old ? 1u : 0u);
    if (h) asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a + 4), "r"(h) : "memory");
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

// Reductions skipped for a zero operand by a predicate on the instruction
// itself, not a branch around it (rows contribute zero words often: the high
// half of a small sum, a count of a valid value).
VR_DEV void s_add_nz(uint64_t* p, uint64_t v) {
    if (v) s_add(p, v);
}
VR_DEV void s_max_nz(uint64_t* p, uint64_t v) {
    asm volatile("{ .reg .pred q; setp.ne.u64 q, %1, 0; @q red.shared.max.u64 [%0], %1; }" ::"r"(smem_u32(p)), "l"(v)
                 : "memory");
}
VR_DEV void s_or_nz(uint64_t* p, uint64_t v) {
    asm volatile("{ .reg .pred q; setp.ne.u64 q, %1, 0; @q red.shared.or.b64 [%0], %1; }" ::"r"(smem_u32(p)), "l"(v)
                 : "memory");
}
VR_DEV void g_add_nz(uint64_t* p, uint64_t v) {
    asm volatile("{ .reg .pred q; setp.ne.u64 q, %1, 0; @q red.relaxed.gpu.global.add.u64 [%0], %1; }" ::"l"(p), "l"(v)
                 : "memory");
}
VR_DEV void g_max_nz(uint64_t* p, uint64_t v) {
    asm volatile("{ .reg .pred q; setp.ne.u64 q, %1, 0; @q red.relaxed.gpu.global.max.u64 [%0], %1; }" ::"l"(p), "l"(v)
                 : "memory");
}
VR_DEV void g_or_nz(uint64_t* p, uint64_t v) {
    asm volatile("{ .reg .pred q; setp.ne.u64 q, %1, 0; @q red.relaxed.gpu.global.or.b64 [%0], %1; }" ::"l"(p), "l"(v)
                 : "memory");
}
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
// 16-byte reads of a two-word key. Not single-copy atomic as a pair: each
// word may be read at a different moment.
VR_DEV void ld2_relaxed_g(const uint64_t* p, uint64_t& a, uint64_t& b) {
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}
VR_DEV void ld2_relaxed_s(const uint64_t* p, uint64_t& a, uint64_t& b) {
    asm volatile("ld.relaxed.cta.shared.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "r"(smem_u32(p)) : "memory");
}

// Address-space dispatch: S = true for shared memory, false for global.
template <bool S> struct Mem;
template <> struct Mem<true> {
    static VR_DEV void add_nz(uint64_t* p, uint64_t v) { s_add_nz(p, v); }
    static VR_DEV void max_nz(uint64_t* p, uint64_t v) { s_max_nz(p, v); }
    static VR_DEV void bor_nz(uint64_t* p, uint64_t v) { s_or_nz(p, v); }
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
    static VR_DEV void ld2(const uint64_t* p, uint64_t& a, uint64_t& b) { ld2_relaxed_s(p, a, b); }
};
template <> struct Mem<false> {
    static VR_DEV void add_nz(uint64_t* p, uint64_t v) { g_add_nz(p, v); }
    static VR_DEV void max_nz(uint64_t* p, uint64_t v) { g_max_nz(p, v); }
    static VR_DEV void bor_nz(uint64_t* p, uint64_t v) { g_or_nz(p, v); }
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
    static VR_DEV void ld2(const uint64_t* p, uint64_t& a, uint64_t& b) { ld2_relaxed_g(p, a, b); }
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

// 10^p for p in [0, 38] as (lo, hi) words, built by the compiler so every
// module (the prebuilt one and each per-spec one) carries its own copy.
struct Pow10Table {
    uint64_t lo[39];
    uint64_t hi[39];
};

constexpr Pow10Table make_pow10_table() {
    Pow10Table t{};
    uint64_t lo = 1, hi = 0;
    for (int i = 0; i < 39; ++i) {
        t.lo[i] = lo;
        t.hi[i] = hi;
        // (hi, lo) *= 10 in 32-bit halves so no 128-bit type is needed
        uint64_t a = (lo & 0xffffffffull) * 10;
        uint64_t b = (lo >> 32) * 10 + (a >> 32);
        lo = (b << 32) | (a & 0xffffffffull);
        hi = hi * 10 + (b >> 32);
    }
    return t;
}

__constant__ const Pow10Table c_pow10 = make_pow10_table();

// |v| < 10^p for a signed 128-bit v (lo, hi).
VR_DEV bool within_precision(uint64_t lo, int64_t hi, int p) {
    uint64_t mlo = lo, mhi = (uint64_t)hi;
    if (hi < 0) {
        mlo = ~lo + 1;
        mhi = ~(uint64_t)hi + (mlo == 0 ? 1 : 0);
    }
    uint64_t plo = c_pow10.lo[p], phi = c_pow10.hi[p];
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
    const int32_t* remap[kMaxCols];  // VR_COL_BATCH_DICTIONARY keys: batch id -> table id
    int32_t remap_n[kMaxCols];
};

// A key id through its batch dictionary's map: the table id, -1 for a null
// entry, -2 for an id outside the batch dictionary.
VR_DEV int32_t remap_id(const TileView& v, int c, uint32_t id) {
    return id < (uint32_t)v.remap_n[c] ? v.remap[c][id] : -2;
}

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

// Loads from a tile the producer staged in shared memory, by 32-bit shared
// address (cheaper than a generic load, which must first find the address
// space). Only for tiles the stage header marks as staged: a batch's last
// partial tile, and batches whose buffers are not 16-byte aligned, are read
// in place from global memory.
VR_DEV int32_t lds32(const void* base, int64_t r) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(base) + (uint32_t)r * 4u;
    int32_t x;
    asm("ld.shared.s32 %0, [%1];" : "=r"(x) : "r"(a));
    return x;
}
VR_DEV int64_t lds64(const void* base, int64_t r) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(base) + (uint32_t)r * 8u;
    int64_t x;
    asm("ld.shared.s64 %0, [%1];" : "=l"(x) : "r"(a));
    return x;
}

// The columns one op reads, with their pointers in registers: built once per
// op per chunk of rows, so the per-row loop reloads nothing from the tile
// header after a store. Column c of the op is 0 (input / first factor),
// 1 (second buffer / factor) or 2 (third factor). SM: the tile's data is
// staged in shared memory (its validity bitmaps may still be global).
template <bool SM>
struct OpViewT {
    const char* d0;
    const char* d1;
    const char* d2;
    const uint32_t* v0;
    const uint32_t* v1;
    const uint32_t* v2;
};
using OpView = OpViewT<false>;
VR_DEV const char* vdata(const TileView& v, int c) { return v.data[c]; }
template <bool SM>
VR_DEV const char* vdata(const OpViewT<SM>& v, int c) { return c == 0 ? v.d0 : c == 1 ? v.d1 : v.d2; }
template <bool SM>
VR_DEV const uint32_t* vvalid(const OpViewT<SM>& v, int c) { return c == 0 ? v.v0 : c == 1 ? v.v1 : v.v2; }
template <bool SM>
VR_DEV bool col_valid(const OpViewT<SM>& v, int c, int64_t r) {
    const uint32_t* w = vvalid(v, c);
    return w == nullptr || bit_at(w, r);
}
template <bool SM>
VR_DEV int32_t ld_i32(const OpViewT<SM>& v, int c, int64_t r) {
    if constexpr (SM) return lds32(vdata(v, c), r);
    return reinterpret_cast<const int32_t*>(vdata(v, c))[r];
}
template <bool SM>
VR_DEV int64_t ld_i64(const OpViewT<SM>& v, int c, int64_t r) {
    if constexpr (SM) return lds64(vdata(v, c), r);
    return reinterpret_cast<const int64_t*>(vdata(v, c))[r];
}
template <bool SM>
VR_DEV double ld_f64(const OpViewT<SM>& v, int c, int64_t r) {
    if constexpr (SM) return __longlong_as_double((long long)lds64(vdata(v, c), r));
    return reinterpret_cast<const double*>(vdata(v, c))[r];
}
template <bool SM>
VR_DEV I128 ld_d128(const OpViewT<SM>& v, int c, int64_t r) {
    I128 x;
    if constexpr (SM) {
        x.lo = (uint64_t)lds64(vdata(v, c), 2 * r);
        x.hi = lds64(vdata(v, c), 2 * r + 1);
    } else {
        const uint64_t* p = reinterpret_cast<const uint64_t*>(vdata(v, c)) + 2 * r;
        x.lo = p[0];
        x.hi = (int64_t)p[1];
    }
    return x;
}
template <bool SM>
VR_DEV int64_t ld_int(const OpViewT<SM>& v, int c, int lane, int64_t r) {
    return lane == VR_INT32 || lane == VR_DICT32 ? (int64_t)ld_i32(v, c, r) : ld_i64(v, c, r);
}

// The op's columns from a tile view; `oo` is `o` with its column indices
// renumbered to the view's 0..2.
template <bool SM>
VR_DEV void make_opview(const OpDesc& o, const TileView& v, OpDesc& oo, OpViewT<SM>& ov) {
    oo = o;
    ov.d0 = ov.d1 = ov.d2 = nullptr;
    ov.v0 = ov.v1 = ov.v2 = nullptr;
    if (o.nterms > 0) {
        ov.d0 = v.data[o.term_col[0]];
        ov.v0 = v.valid[o.term_col[0]];
        ov.d1 = v.data[o.term_col[1]];
        ov.v1 = v.valid[o.term_col[1]];
        if (o.nterms > 2) {
            ov.d2 = v.data[o.term_col[2]];
            ov.v2 = v.valid[o.term_col[2]];
        }
        oo.term_col[0] = 0;
        oo.term_col[1] = 1;
        oo.term_col[2] = 2;
    } else if (o.col >= 0) {
        ov.d0 = v.data[o.col];
        ov.v0 = v.valid[o.col];
        oo.col = 0;
        if (o.col2 >= 0) {
            ov.d1 = v.data[o.col2];
            ov.v1 = v.valid[o.col2];
            oo.col2 = 1;
        }
    }
}

// ------------------------------------------------------ key packing ----
// k[idx] |= v with a runtime idx, without indexing the array at run time
// (which would place it in local memory).
template <int KW>
VR_DEV void or_word(uint64_t (&k)[KW], int idx, uint64_t v) {
#pragma unroll
    for (int i = 0; i < KW; ++i)
        if (i == idx) k[i] |= v;
}

// Packs row r's key tuple into KW words; `side` is set for the one single
// 64-bit key equal to kSentinel (sentinel layout only). Null keys store zero
// data and their null bit, as GroupKeyTable.insert does (GroupKeyTable.java:2515-2540).
// One key field of row r into the packed words (null: its null bit only).
template <int KW>
VR_DEV void pack_field(const KeyField& kf, const TileView& v, int64_t r, uint64_t (&k)[KW], bool& bad) {
    if (kf.null_word >= 0 && !col_valid(v, kf.col, r)) {  // only nullable keys carry a bitmap
        or_word<KW>(k, kf.null_word, 1ull << kf.null_shift);
        return;
    }
    switch (kf.lane) {
        case VR_INT32:
        case VR_DICT32: {
            uint32_t u = (uint32_t)ld_i32(v, kf.col, r);
            if (kf.remap) {  // the batch's dictionary id -> the table's
                const int32_t t = remap_id(v, kf.col, u);
                if (t == -1) {  // a null entry: the row's key is null (GroupKeyTable.java:1388-1389)
                    if (kf.null_word >= 0)
                        or_word<KW>(k, kf.null_word, 1ull << kf.null_shift);
                    else
                        bad = true;
                    return;
                }
                if (t < 0) bad = true;
                u = (uint32_t)(t < 0 ? 0 : t);
            }
            if (kf.bits < 32 && (u >> kf.bits) != 0) bad = true;  // id outside the declared dictionary
            or_word<KW>(k, kf.word, (uint64_t)u << kf.shift);
            break;
        }
        case VR_INT64:
        case VR_FLOAT64:
            or_word<KW>(k, kf.word, ld_u64(v, kf.col, r));
            break;
        case VR_BOOL:
            or_word<KW>(k, kf.word, (uint64_t)bit_at(reinterpret_cast<const uint32_t*>(v.data[kf.col]), r) << kf.shift);
            break;
        case VR_DECIMAL128: {
            I128 x = ld_d128(v, kf.col, r);
            or_word<KW>(k, kf.word, x.lo);
            or_word<KW>(k, kf.word + 1, (uint64_t)x.hi);
            break;
        }
    }
}

// The occupancy bit, or (sentinel layout: one 64-bit word, no spare bit) the
// xor with kSentinel and the side-slot test.
template <int KW>
VR_DEV void pack_finish(int occ_word, int occ_shift, uint64_t (&k)[KW], bool& side) {
    if (occ_word >= 0) {
        or_word<KW>(k, occ_word, 1ull << occ_shift);
    } else {
        side = (k[0] == kSentinel);
        k[0] ^= kSentinel;
    }
}

template <int KW>
VR_DEV void pack_key(const Program& P, const TileView& v, int64_t r, uint64_t (&k)[KW], bool& side, bool& bad) {
#pragma unroll
    for (int i = 0; i < KW; ++i) k[i] = 0;
    side = false;
    bad = false;
    for (int f = 0; f < P.num_keys; ++f) pack_field<KW>(P.keys[f], v, r, k, bad);
    pack_finish<KW>(P.occ_word, P.occ_shift, k, side);
}

// Direct tier: one field's share of the combination index; -1 when its id
// lies outside the declared dictionary (null is the field's last value).
template <bool SM = false>
VR_DEV int64_t direct_field(const KeyField& kf, const TileView& v, int64_t r) {
    int64_t val;
    if (kf.null_word >= 0 && !col_valid(v, kf.col, r)) {  // only nullable keys carry a bitmap
        val = kf.card - 1;
    } else if (kf.lane == VR_BOOL) {
        val = bit_at(reinterpret_cast<const uint32_t*>(v.data[kf.col]), r);
    } else {
        val = (int64_t)(uint32_t)(SM ? lds32(v.data[kf.col], r) : ld_i32(v, kf.col, r));
        if (kf.remap) {
            const int32_t t = remap_id(v, kf.col, (uint32_t)val);
            if (t == -1 && kf.null_word >= 0) return (int64_t)(kf.card - 1) * kf.mul;  // a null entry
            if (t < 0) return -1;
            val = t;
        }
        if (val >= (int64_t)kf.card - (kf.null_word >= 0 ? 1 : 0)) return -1;
    }
    return val * kf.mul;
}

// direct_field in 32-bit arithmetic (a combination index is below 65,536).
template <bool SM>
VR_DEV int direct_field32(const KeyField& kf, const TileView& v, int64_t r) {
    int val;
    if (kf.null_word >= 0 && !col_valid(v, kf.col, r)) {
        val = (int)kf.card - 1;
    } else if (kf.lane == VR_BOOL) {
        val = (int)bit_at(reinterpret_cast<const uint32_t*>(v.data[kf.col]), r);
    } else {
        uint32_t id = (uint32_t)(SM ? lds32(v.data[kf.col], r) : ld_i32(v, kf.col, r));
        if (kf.remap) {
            const int32_t t = remap_id(v, kf.col, id);
            if (t == -1 && kf.null_word >= 0) return ((int)kf.card - 1) * (int)kf.mul;  // a null entry
            id = t < 0 ? 0xffffffffu : (uint32_t)t;
        }
        if (id >= (uint32_t)kf.card - (kf.null_word >= 0 ? 1u : 0u)) return -1;
        val = (int)id;
    }
    return val * (int)kf.mul;
}

// Direct tier: the combination index of a row's dictionary / boolean keys;
// -1 when an id lies outside its declared dictionary.
VR_DEV int64_t direct_index(const Program& P, const TileView& v, int64_t r) {
    int64_t idx = 0;
    for (int f = 0; f < P.num_keys; ++f) {
        int64_t x = direct_field(P.keys[f], v, r);
        if (x < 0) return -1;
        idx += x;
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
//   KW == 2 (slots 16-byte aligned: the slot width is even): one 128-bit CAS
//     from 0 claims and publishes the whole key (the occupancy bit is in the
//     last word, so a published key is never 0). A slot changes once, from 0
//     to its key, so any non-zero word a plain 16-byte read returns is final;
//     a zero word may be stale, and only then does the probe fall back to the
//     CAS, which inserts or returns the slot's true content. No fence, no
//     lock (an acquire per probe and a release per insert cost 12-17% on
//     20M rows into 4M two-word groups).
//   KW >= 3: claim the last word with a BUSY bit, write the other words,
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
        } else if (KW == 2) {
            uint64_t w0, w1;
            Mem<S>::ld2(slot, w0, w1);
            if (w0 != 0 && w1 != 0) {  // both words final
                if (w0 == k[0] && w1 == k[KW - 1]) return slot;
            } else if (w1 == 0 || w1 == k[KW - 1]) {  // empty, or a zero word that may be stale
                uint64_t c0 = 0, c1 = 0;
                if (Mem<S>::cas128(slot, c0, c1, k[0], k[KW - 1])) {
                    fresh = true;
                    return slot;
                }
                if (c0 == k[0] && c1 == k[KW - 1]) return slot;
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
// One row's contribution to an op, held in registers: the eight words are
// named fields and are only ever addressed statically (an array indexed by a
// runtime word count would live in local memory, which with most of L1
// carved out for shared memory goes to L2).
//
// Three representations (words relative to the op's first word):
//   raw     - values as read from the row (op_raw);
//   global  - the shared/HBM table words: carry-save limbs that add exactly
//             with 64-bit atomics, in any order (raw_to_global);
//   private - the direct tier's thread-private words: running 64/128-bit sums
//             plus a wrap count, so a sum touches one or two words per row.
// kind         global words                           private words
// COUNT_*      a=count                                a=count
// SUM_I32      a=sum                                  a=sum
// SUM_I64      a=sum of lo32 (s) b=sum of hi32 (s)    a=int64 sum  b=wraps
// SUM_F64      a=sum b=compensation                   a=sum b=compensation
// SUM_D128     a..d=32-bit limbs (d signed)           a,b=int128 sum  c=wraps
// SUM_PROD     a,b=cs  c..f=limbs  g=ANSI flag        a=int64 sum b=wraps c,d=int128 e=wraps
//              h=null products                        g=flag h=null products
// MAX_KEY      a                                      a
// MAX_D128     a=lo b=hi                              a=lo b=hi
// MERGE_DSUM   a..d=limbs e=flags                     a,b=int128 c=wraps e=flags
// MERGE_DAVG   a..d=limbs e,f=count cs g=flags        a,b=int128 c=wraps e=count f=wraps g=flags
struct Contrib {
    uint64_t a, b, c, d, e, f, g, h;
};

VR_DEV void czero(Contrib& x) { x.a = x.b = x.c = x.d = x.e = x.f = x.g = x.h = 0; }
VR_DEV uint64_t hi32(int64_t x) { return (uint64_t)(int64_t)(int32_t)(x >> 32); }
// Signed carry-save split of an int64: x = lo + hi * 2^32 with lo the
// sign-extended low 32 bits, so |x| < 2^31 has hi == 0 (one atomic, not two).
// Table words accumulate lo and hi parts; a low word's total is read signed.
VR_DEV void split_cs(int64_t x, uint64_t& lo, uint64_t& hi) {
    const int64_t l = (int64_t)(int32_t)x;
    lo = (uint64_t)l;
    hi = (uint64_t)((x >> 32) + (l < 0 ? 1 : 0));
}

// Validity of input column c of op o at row r: only columns the spec
// declares nullable are tested (a non-nullable column never carries a bitmap).
template <class V>
VR_DEV bool in_valid(const OpDesc& o, const V& v, int c, int64_t r) {
    return !(o.flags & OPF_NULLABLE) || col_valid(v, c, r);
}

// |p| < 10^prec for an int64 p (2^63 < 10^19: always true from 19 digits on).
VR_DEV bool within_precision64(int64_t p, int prec) {
    if (prec >= 19) return true;
    const uint64_t m = p < 0 ? 0ull - (uint64_t)p : (uint64_t)p;
    return m < c_pow10.lo[prec];
}

// The exact product a * b * c (c = 1 for two factors) of a decimal
// product row whose int64 fast path gave up: int64, 128-bit, or null (past
// 128 bits or the precision; `error` with ANSI). Out of line: rare rows.
struct ProdResult {
    enum { kInt64 = 0, kWide = 1, kNull = 2 };
    uint64_t lo, hi;
    uint32_t kind, error;
};
static __device__ __noinline__ ProdResult product_exact(int64_t a, int64_t b, int64_t c, int prec, bool checked) {
    ProdResult s = {0, 0, ProdResult::kNull, checked ? 1u : 0u};
    I128 p = mul_i64(a, b);
    if (c != 1) {
        I128 q;
        if (!mul_i128_i64(p, c, q)) return s;
        p = q;
    }
    if (!within_precision(p.lo, p.hi, prec)) return s;
    s.error = 0;
    s.lo = p.lo;
    s.hi = (uint64_t)p.hi;
    s.kind = p.hi == ((int64_t)p.lo >> 63) ? ProdResult::kInt64 : ProdResult::kWide;
    return s;
}

template <class V>
VR_DEV bool terms_valid(const OpDesc& o, const V& v, int64_t r) {
    bool ok = in_valid(o, v, o.term_col[0], r) && in_valid(o, v, o.term_col[1], r);
    if (o.nterms > 2) ok = ok && in_valid(o, v, o.term_col[2], r);
    return ok;
}

template <class V>
VR_DEV int64_t term_value(const OpDesc& o, const V& v, int64_t r, int t) {
    int64_t x = ld_i64(v, o.term_col[t], r);
    return o.term_add[t] + (o.term_sign[t] < 0 ? -x : x);
}

// Raw values of row r for op o; false when the row contributes nothing.
template <int K, class V>
VR_DEV bool op_raw(const OpDesc& o, const V& v, int64_t r, Contrib& x) {
    czero(x);
    switch (K) {
        case OP_COUNT_ROWS:
            x.a = 1;
            return true;
        case OP_COUNT_VALID: {
            bool ok = o.nterms > 0 ? terms_valid(o, v, r) : in_valid(o, v, o.col, r);
            x.a = ok ? 1 : 0;
            return ok;
        }
        case OP_SUM_I32:
            if (!in_valid(o, v, o.col, r)) return false;
            x.a = (uint64_t)(int64_t)ld_i32(v, o.col, r);
            return true;
        case OP_SUM_I64:
            if (!in_valid(o, v, o.col, r)) return false;
            x.a = (uint64_t)ld_int(v, o.col, o.lane, r);
            return true;
        case OP_SUM_F64:
            if (!in_valid(o, v, o.col, r)) return false;
            x.a = (uint64_t)__double_as_longlong(ld_f64(v, o.col, r));
            return true;
        case OP_SUM_D128: {
            if (!in_valid(o, v, o.col, r)) return false;
            I128 d = ld_d128(v, o.col, r);
            x.a = d.lo;
            x.b = (uint64_t)d.hi;
            return true;
        }
        case OP_SUM_PROD: {
            if (!terms_valid(o, v, r)) {
                x.h = 1;  // a null factor: the product is null
                return true;
            }
            // Fast path: every partial product fits int64 (mul.lo's sign
            // extension equals mul.hi) and lies within the precision; other
            // rows take the exact 128-bit path out of line.
            const int64_t a = term_value(o, v, r, 0), b = term_value(o, v, r, 1);
            int64_t p = a * b;
            bool fits = __mul64hi(a, b) == (p >> 63);
            int64_t c = 1;
            if (o.nterms == 3) {
                c = term_value(o, v, r, 2);
                const int64_t q = p * c;
                fits = fits && __mul64hi(p, c) == (q >> 63);
                p = q;
            }
            if (fits && within_precision64(p, o.prec)) {
                x.a = (uint64_t)p;
                return true;
            }
            const ProdResult s = product_exact(a, b, c, o.prec, (o.flags & OPF_CHECKED) != 0);
            if (s.kind == ProdResult::kNull) {
                // Spark's CheckOverflow on the product: null (non-ANSI) or an error (ANSI)
                x.h = 1;
                x.g = s.error;
            } else if (s.kind == ProdResult::kInt64) {
                x.a = s.lo;
            } else {
                x.c = s.lo;
                x.d = s.hi;
                x.e = 1;  // marks the 128-bit case in the raw form
            }
            return true;
        }
        case OP_MAX_KEY: {
            if (!in_valid(o, v, o.col, r)) return false;
            uint64_t k = o.lane == VR_FLOAT64 ? okey_f64(ld_f64(v, o.col, r)) : okey_i64(ld_int(v, o.col, o.lane, r));
            x.a = (o.flags & OPF_MIN) ? ~k : k;
            return true;
        }
        case OP_MAX_D128: {
            if (!in_valid(o, v, o.col, r)) return false;
            I128 d = ld_d128(v, o.col, r);
            uint64_t lo = d.lo, hi = (uint64_t)d.hi ^ 0x8000000000000000ull;
            if (o.flags & OPF_MIN) {
                lo = ~lo;
                hi = ~hi;
            }
            x.a = lo;
            x.b = hi;
            return true;
        }
        case OP_MERGE_DSUM: {
            // WideDecimalSumMergeAgg.merge (VectorAggregates.scala:700-725): rows whose isEmpty is
            // null or true are skipped; a null sum on a non-empty row poisons the group.
            if (!in_valid(o, v, o.col2, r) || bit_at(reinterpret_cast<const uint32_t*>(vdata(v, o.col2)), r)) return false;
            if (!in_valid(o, v, o.col, r)) {
                x.e = kFlagNonEmpty | kFlagOverflow;
                return true;
            }
            I128 d = ld_d128(v, o.col, r);
            x.a = d.lo;
            x.b = (uint64_t)d.hi;
            x.e = kFlagNonEmpty;
            return true;
        }
        case OP_MERGE_DAVG: {
            // WideDecimalAvgMergeAgg.merge (VectorAggregates.scala:557-573): counts add when valid;
            // a null sum poisons the group.
            if (in_valid(o, v, o.col2, r)) x.e = (uint64_t)ld_i64(v, o.col2, r);
            if (!in_valid(o, v, o.col, r)) {
                x.g = kFlagOverflow;
                return true;
            }
            I128 d = ld_d128(v, o.col, r);
            x.a = d.lo;
            x.b = (uint64_t)d.hi;
            return true;
        }
    }
    return false;
}

// 128-bit value (lo, hi) as four 32-bit carry-save limbs (limb 3 signed).
VR_DEV void limbs_of(uint64_t lo, uint64_t hi, uint64_t& l0, uint64_t& l1, uint64_t& l2, uint64_t& l3) {
    l0 = (uint32_t)lo;
    l1 = lo >> 32;
    l2 = (uint32_t)hi;
    l3 = hi32((int64_t)hi);
}

// raw -> global representation, in place.
template <int K>
VR_DEV void raw_to_global(const OpDesc& o, Contrib& x) {
    (void)o;
    switch (K) {
        case OP_SUM_I64:
            split_cs((int64_t)x.a, x.a, x.b);
            break;
        case OP_SUM_D128:
            limbs_of(x.a, x.b, x.a, x.b, x.c, x.d);
            break;
        case OP_SUM_PROD:
            if (x.e) {
                uint64_t lo = x.c, hi = x.d;
                x.a = x.b = 0;
                limbs_of(lo, hi, x.c, x.d, x.e, x.f);
            } else {
                split_cs((int64_t)x.a, x.a, x.b);
            }
            break;
        case OP_MERGE_DSUM:
            limbs_of(x.a, x.b, x.a, x.b, x.c, x.d);
            break;
        case OP_MERGE_DAVG: {
            int64_t n = (int64_t)x.e;
            limbs_of(x.a, x.b, x.a, x.b, x.c, x.d);
            split_cs(n, x.e, x.f);
            break;
        }
        default:
            break;
    }
}

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
VR_DEV double as_f64(uint64_t u) { return __longlong_as_double((long long)u); }
VR_DEV uint64_t as_u64(double d) { return (uint64_t)__double_as_longlong(d); }

// ------------------------------------------------ warp peer reduction ----
// Peers are lanes holding the same key (from __match_any_sync). A tree over
// each peer group's ranks: at step s the lane of rank r (r % 2^(s+1) == 0)
// takes the partial of rank r + 2^s. The lowest lane ends with the total.
VR_DEV int nth_set_bit(uint32_t mask, int n) {
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
    int src0, src1, src2, src3, src4;
    uint32_t recv;  // bit s: this lane adds the partial it receives at step s
};

VR_DEV PeerPlan make_peer_plan(uint32_t peers, int lane) {
    PeerPlan pp;
    int n = __popc(peers);
    int r = __popc(peers & ((1u << lane) - 1u));
    int maxn = (int)__reduce_max_sync(kFull, (unsigned)n);
    pp.steps = 0;
    while ((1 << pp.steps) < maxn) ++pp.steps;
    pp.recv = 0;
    int src[5];
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        src[s] = lane;
        int stride = 1 << s;
        if (s < pp.steps && (r % (2 * stride)) == 0 && r + stride < n) {
            pp.recv |= 1u << s;
            src[s] = nth_set_bit(peers, r + stride);
        }
    }
    pp.src0 = src[0];
    pp.src1 = src[1];
    pp.src2 = src[2];
    pp.src3 = src[3];
    pp.src4 = src[4];
    return pp;
}

VR_DEV int pp_src(const PeerPlan& pp, int s) {
    return s == 0 ? pp.src0 : s == 1 ? pp.src1 : s == 2 ? pp.src2 : s == 3 ? pp.src3 : pp.src4;
}

enum RedKind { R_ADD, R_MAX, R_OR };

template <int K>
VR_DEV uint64_t red1(const PeerPlan& pp, uint64_t x) {
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        if (s < pp.steps) {
            uint64_t t = (uint64_t)__shfl_sync(kFull, (unsigned long long)x, pp_src(pp, s));
            if (pp.recv & (1u << s)) x = K == R_ADD ? x + t : K == R_MAX ? (t > x ? t : x) : (x | t);
        }
    }
    return x;
}

VR_DEV void red_dd(const PeerPlan& pp, uint64_t& s_bits, uint64_t& c_bits) {
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        if (s < pp.steps) {
            uint64_t ts = (uint64_t)__shfl_sync(kFull, (unsigned long long)s_bits, pp_src(pp, s));
            uint64_t tc = (uint64_t)__shfl_sync(kFull, (unsigned long long)c_bits, pp_src(pp, s));
            if (pp.recv & (1u << s)) {
                double a = as_f64(s_bits), c = as_f64(c_bits);
                dd_add(a, c, as_f64(ts), as_f64(tc));
                s_bits = as_u64(a);
                c_bits = as_u64(c);
            }
        }
    }
}

VR_DEV void red_max128(const PeerPlan& pp, uint64_t& lo, uint64_t& hi) {
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        if (s < pp.steps) {
            uint64_t tl = (uint64_t)__shfl_sync(kFull, (unsigned long long)lo, pp_src(pp, s));
            uint64_t th = (uint64_t)__shfl_sync(kFull, (unsigned long long)hi, pp_src(pp, s));
            if ((pp.recv & (1u << s)) && u128_gt(tl, th, lo, hi)) {
                lo = tl;
                hi = th;
            }
        }
    }
}

// Combines the global-representation contribution over each peer group.
template <int K>
VR_DEV void peer_reduce(const OpDesc& o, const PeerPlan& pp, Contrib& x) {
    (void)o;
    switch (K) {
        case OP_COUNT_ROWS:
        case OP_COUNT_VALID:
        case OP_SUM_I32:
            x.a = red1<R_ADD>(pp, x.a);
            break;
        case OP_SUM_I64:
            x.a = red1<R_ADD>(pp, x.a);
            x.b = red1<R_ADD>(pp, x.b);
            break;
        case OP_SUM_F64:
            red_dd(pp, x.a, x.b);
            break;
        case OP_SUM_D128:
        case OP_MERGE_DSUM:
        case OP_MERGE_DAVG:
            x.a = red1<R_ADD>(pp, x.a);
            x.b = red1<R_ADD>(pp, x.b);
            x.c = red1<R_ADD>(pp, x.c);
            x.d = red1<R_ADD>(pp, x.d);
            if (K == OP_MERGE_DSUM) {
                x.e = red1<R_OR>(pp, x.e);
            } else if (K == OP_MERGE_DAVG) {
                x.e = red1<R_ADD>(pp, x.e);
                x.f = red1<R_ADD>(pp, x.f);
                x.g = red1<R_OR>(pp, x.g);
            }
            break;
        case OP_SUM_PROD: {
            x.a = red1<R_ADD>(pp, x.a);
            x.b = red1<R_ADD>(pp, x.b);
            if (__any_sync(kFull, (x.c | x.d | x.e | x.f | x.g) != 0)) {  // rare: 128-bit products, errors
                x.c = red1<R_ADD>(pp, x.c);
                x.d = red1<R_ADD>(pp, x.d);
                x.e = red1<R_ADD>(pp, x.e);
                x.f = red1<R_ADD>(pp, x.f);
                x.g = red1<R_OR>(pp, x.g);
            }
            x.h = red1<R_ADD>(pp, x.h);
            break;
        }
        case OP_MAX_KEY:
            x.a = red1<R_MAX>(pp, x.a);
            break;
        case OP_MAX_D128:
            red_max128(pp, x.a, x.b);
            break;
    }
}

// ----------------------------------------------------- atomic apply ----
template <bool S>
VR_DEV void add_nz(uint64_t* p, uint64_t v) {
    Mem<S>::add_nz(p, v);
}
template <bool S>
VR_DEV void or_nz(uint64_t* p, uint64_t v) {
    Mem<S>::bor_nz(p, v);
}
template <bool S>
VR_DEV void max_nz(uint64_t* p, uint64_t v) {
    if (S) {
        // A max only grows, so a value not above a (possibly stale) read of
        // it cannot change it: after the first rows nearly every row skips
        // its shared-memory atomic. HBM words keep the plain reduction (a
        // read there is a round trip).
        if (v <= *(const volatile uint64_t*)p) return;
    }
    Mem<S>::max_nz(p, v);
}
// Compensated atomic add of a double-double (s, c): the hardware add rounds to
// nearest like __dadd_rn, so the thread recovers the exact rounding error of
// its own add and accumulates it (with the incoming compensation) in the next word.
template <bool S>
VR_DEV void fadd_pair(uint64_t* p, uint64_t s_bits, uint64_t c_bits) {
    if (!(s_bits | c_bits)) return;
    double s = as_f64(s_bits), cc = as_f64(c_bits);
    double old = Mem<S>::fadd(reinterpret_cast<double*>(p), s);
    double nw, err;
    two_sum(old, s, nw, err);
    double tot = __dadd_rn(err, cc);
    if (tot != 0.0) Mem<S>::fadd(reinterpret_cast<double*>(p + 1), tot);
}
template <bool S>
VR_DEV void max128(uint64_t* p, uint64_t lo, uint64_t hi) {
    if (!(lo | hi)) return;
    uint64_t clo = Mem<S>::ld(p), chi = Mem<S>::ld(p + 1);
    for (int it = 0; it < (1 << 16) && u128_gt(lo, hi, clo, chi); ++it)
        if (Mem<S>::cas128(p, clo, chi, lo, hi)) break;
}

// Applies a global-representation contribution to the op's words at `acc`.
template <int K, bool S>
VR_DEV void apply_global(const OpDesc& o, uint64_t* acc, const Contrib& x) {
    (void)o;
    switch (K) {
        case OP_COUNT_ROWS:
        case OP_COUNT_VALID:
        case OP_SUM_I32:
            add_nz<S>(acc, x.a);
            break;
        case OP_SUM_I64:
            add_nz<S>(acc, x.a);
            add_nz<S>(acc + 1, x.b);
            break;
        case OP_SUM_F64:
            fadd_pair<S>(acc, x.a, x.b);
            break;
        case OP_SUM_D128:
            add_nz<S>(acc, x.a);
            add_nz<S>(acc + 1, x.b);
            add_nz<S>(acc + 2, x.c);
            add_nz<S>(acc + 3, x.d);
            break;
        case OP_SUM_PROD:
            add_nz<S>(acc, x.a);
            add_nz<S>(acc + 1, x.b);
            add_nz<S>(acc + 2, x.c);
            add_nz<S>(acc + 3, x.d);
            add_nz<S>(acc + 4, x.e);
            add_nz<S>(acc + 5, x.f);
            or_nz<S>(acc + 6, x.g);
            add_nz<S>(acc + 7, x.h);
            break;
        case OP_MAX_KEY:
            max_nz<S>(acc, x.a);
            break;
        case OP_MAX_D128:
            max128<S>(acc, x.a, x.b);
            break;
        case OP_MERGE_DSUM:
            add_nz<S>(acc, x.a);
            add_nz<S>(acc + 1, x.b);
            add_nz<S>(acc + 2, x.c);
            add_nz<S>(acc + 3, x.d);
            or_nz<S>(acc + 4, x.e);
            break;
        case OP_MERGE_DAVG:
            add_nz<S>(acc, x.a);
            add_nz<S>(acc + 1, x.b);
            add_nz<S>(acc + 2, x.c);
            add_nz<S>(acc + 3, x.d);
            add_nz<S>(acc + 4, x.e);
            add_nz<S>(acc + 5, x.f);
            or_nz<S>(acc + 6, x.g);
            break;
    }
}

// Compile-time op kinds: dispatch_kind(kind, f) calls f(KindTag<K>{}) with the
// runtime kind as a constant, so per-kind code folds its switches away.
template <int K>
struct KindTag {
    static constexpr int value = K;
};
template <class F>
VR_DEV void dispatch_kind(int kind, F&& f) {
    switch (kind) {
        case OP_COUNT_ROWS: f(KindTag<OP_COUNT_ROWS>{}); break;
        case OP_COUNT_VALID: f(KindTag<OP_COUNT_VALID>{}); break;
        case OP_SUM_I32: f(KindTag<OP_SUM_I32>{}); break;
        case OP_SUM_I64: f(KindTag<OP_SUM_I64>{}); break;
        case OP_SUM_F64: f(KindTag<OP_SUM_F64>{}); break;
        case OP_SUM_D128: f(KindTag<OP_SUM_D128>{}); break;
        case OP_SUM_PROD: f(KindTag<OP_SUM_PROD>{}); break;
        case OP_MAX_KEY: f(KindTag<OP_MAX_KEY>{}); break;
        case OP_MAX_D128: f(KindTag<OP_MAX_D128>{}); break;
        case OP_MERGE_DSUM: f(KindTag<OP_MERGE_DSUM>{}); break;
        case OP_MERGE_DAVG: f(KindTag<OP_MERGE_DAVG>{}); break;
    }
}

// Loads an op's global-representation state (a table slot's words) so it can
// be applied to another table (shared-tier flush, rehash, spill merge).
VR_DEV void load_state(const OpDesc& o, const uint64_t* acc, Contrib& x) {
    czero(x);
    int n = o.nwords;
    x.a = acc[0];
    if (n > 1) x.b = acc[1];
    if (n > 2) x.c = acc[2];
    if (n > 3) x.d = acc[3];
    if (n > 4) x.e = acc[4];
    if (n > 5) x.f = acc[5];
    if (n > 6) x.g = acc[6];
    if (n > 7) x.h = acc[7];
}

// ------------------------------------------------ thread-private apply ----
// Direct tier: each consumer thread keeps an op's hot words (the running
// values every row touches) privately, word i at hot[i * stride]; rare
// events (64/128-bit wraps, 128-bit products, null products, error flags)
// go with shared-memory atomics into a per-CTA copy of the op's global words
// (`cold`). Hot words per kind: 1, except SUM_F64 / SUM_D128 / MAX_D128 (2:
// sum+compensation, lo+hi) and MERGE_DSUM / MERGE_DAVG (3: lo, hi, flags or count).

// hot += v; a signed wrap adds +-2^64 to the cold carry-save high word (+-2^32 there).
VR_DEV void hot_add_i64(uint64_t* hot, uint64_t* cold_hi, int64_t v) {
    int64_t s = (int64_t)*hot;
    int64_t ns = (int64_t)((uint64_t)s + (uint64_t)v);
    if (((s ^ ns) & (v ^ ns)) < 0) s_add(cold_hi, v > 0 ? (1ull << 32) : (0ull - (1ull << 32)));
    *hot = (uint64_t)ns;
}
// (lo, hi) += (xlo, xhi) as int128; a wrap adds +-2^128 to the cold limb 3 (+-2^32 there).
VR_DEV void hot_add_i128(uint64_t* lo, uint64_t* hi, uint64_t* cold_l3, uint64_t xlo, uint64_t xhi) {
    uint64_t l = *lo, h = *hi;
    uint64_t nl = l + xlo;
    uint64_t nh = h + xhi + (nl < l ? 1 : 0);
    if ((int64_t)((h ^ nh) & (xhi ^ nh)) < 0) s_add(cold_l3, (int64_t)xhi >= 0 ? (1ull << 32) : (0ull - (1ull << 32)));
    *lo = nl;
    *hi = nh;
}

template <int K>
VR_DEV void apply_private(const OpDesc& o, uint64_t* hot, int stride, uint64_t* cold, const Contrib& x) {
    (void)o;
    switch (K) {
        case OP_COUNT_ROWS:
        case OP_COUNT_VALID:
        case OP_SUM_I32:
            hot[0] += x.a;
            break;
        case OP_SUM_I64:
            hot_add_i64(hot, cold + 1, (int64_t)x.a);
            break;
        case OP_SUM_F64: {
            double s = as_f64(hot[0]), c = as_f64(hot[stride]), v = as_f64(x.a);
            double t = __dadd_rn(s, v);
            if (isfinite(t))
                c = __dadd_rn(c, fabs(s) >= fabs(v) ? __dadd_rn(__dsub_rn(s, t), v) : __dadd_rn(__dsub_rn(v, t), s));
            hot[0] = as_u64(t);
            hot[stride] = as_u64(c);
            break;
        }
        case OP_SUM_D128:
            hot_add_i128(hot, hot + stride, cold + 3, x.a, x.b);
            break;
        case OP_SUM_PROD:
            if (x.h) {
                s_add(cold + 7, 1);
                if (x.g) s_or(cold + 6, 1);
            } else if (x.e) {
                uint64_t l0, l1, l2, l3;
                limbs_of(x.c, x.d, l0, l1, l2, l3);
                s_add(cold + 2, l0);
                s_add(cold + 3, l1);
                s_add(cold + 4, l2);
                s_add(cold + 5, l3);
            } else {
                hot_add_i64(hot, cold + 1, (int64_t)x.a);
            }
            break;
        case OP_MAX_KEY:
            if (x.a > hot[0]) hot[0] = x.a;
            break;
        case OP_MAX_D128:
            if (u128_gt(x.a, x.b, hot[0], hot[stride])) {
                hot[0] = x.a;
                hot[stride] = x.b;
            }
            break;
        case OP_MERGE_DSUM:
            hot[2 * stride] |= x.e;
            if (x.a | x.b) hot_add_i128(hot, hot + stride, cold + 3, x.a, x.b);
            break;
        case OP_MERGE_DAVG:
            if (x.e) hot_add_i64(hot + 2 * stride, cold + 5, (int64_t)x.e);
            if (x.g) s_or(cold + 6, x.g);
            if (x.a | x.b) hot_add_i128(hot, hot + stride, cold + 3, x.a, x.b);
            break;
    }
}

// ----------------------------------------------- private -> global flush ----
// A signed 192-bit accumulator (lo: 128 bits, hi: the rest) for exact sums of
// thread-private partials.
struct Acc192 {
    unsigned __int128 lo;
    int64_t hi;
};
VR_DEV void acc_zero(Acc192& a) {
    a.lo = 0;
    a.hi = 0;
}
VR_DEV void acc_add_i128(Acc192& a, uint64_t xlo, uint64_t xhi) {
    unsigned __int128 x = ((unsigned __int128)xhi << 64) | xlo;
    unsigned __int128 n = a.lo + x;
    a.hi += (n < a.lo ? 1 : 0) + ((int64_t)xhi < 0 ? -1 : 0);
    a.lo = n;
}
VR_DEV void acc_add_i64(Acc192& a, int64_t v) { acc_add_i128(a, (uint64_t)v, v < 0 ? ~0ull : 0ull); }
// Global carry-save words (lo32 unsigned, rest signed) that add the value.
VR_DEV void acc_to_cs(const Acc192& a, uint64_t& w0, uint64_t& w1) {
    w0 = (uint32_t)a.lo;
    w1 = (uint64_t)(a.lo >> 32);  // exact while |value| < 2^95
}
VR_DEV void acc_to_limbs(const Acc192& a, uint64_t& l0, uint64_t& l1, uint64_t& l2, uint64_t& l3) {
    l0 = (uint32_t)a.lo;
    l1 = (uint32_t)(a.lo >> 32);
    l2 = (uint32_t)(a.lo >> 64);
    l3 = (uint64_t)(((int64_t)a.hi << 32) | (int64_t)(uint64_t)(a.lo >> 96));  // value >> 96, |value| < 2^159
}

// Combines the hot words of one op over all nt consumer threads (word i of
// thread t at hot[i * nt + t]) into a global-representation contribution.
template <int K>
VR_DEV void private_to_global(const OpDesc& o, const uint64_t* hot, int nt, Contrib& x) {
    (void)o;
    czero(x);
    const int64_t S = nt;
    switch (K) {
        case OP_COUNT_ROWS:
        case OP_COUNT_VALID:
        case OP_SUM_I32:
            #pragma unroll 1  // once per CTA: keep it small
            for (int t = 0; t < nt; ++t) x.a += hot[t];
            break;
        case OP_MAX_KEY:
            #pragma unroll 1  // once per CTA: keep it small
            for (int t = 0; t < nt; ++t) x.a = hot[t] > x.a ? hot[t] : x.a;
            break;
        case OP_MAX_D128:
            #pragma unroll 1  // once per CTA: keep it small
            for (int t = 0; t < nt; ++t)
                if (u128_gt(hot[t], hot[S + t], x.a, x.b)) {
                    x.a = hot[t];
                    x.b = hot[S + t];
                }
            break;
        case OP_SUM_F64: {
            double s = 0.0, c = 0.0;
            #pragma unroll 1  // once per CTA: keep it small
            for (int t = 0; t < nt; ++t) dd_add(s, c, as_f64(hot[t]), as_f64(hot[S + t]));
            x.a = as_u64(s);
            x.b = as_u64(c);
            break;
        }
        case OP_SUM_I64:
        case OP_SUM_PROD: {
            Acc192 a;
            acc_zero(a);
            #pragma unroll 1  // once per CTA: keep it small
            for (int t = 0; t < nt; ++t) acc_add_i64(a, (int64_t)hot[t]);
            acc_to_cs(a, x.a, x.b);
            break;
        }
        case OP_SUM_D128:
        case OP_MERGE_DSUM:
        case OP_MERGE_DAVG: {
            Acc192 a;
            acc_zero(a);
            #pragma unroll 1  // once per CTA: keep it small
            for (int t = 0; t < nt; ++t) acc_add_i128(a, hot[t], hot[S + t]);
            acc_to_limbs(a, x.a, x.b, x.c, x.d);
            if (K == OP_MERGE_DSUM) {
                #pragma unroll 1  // once per CTA: keep it small
                for (int t = 0; t < nt; ++t) x.e |= hot[2 * S + t];
            } else if (K == OP_MERGE_DAVG) {
                Acc192 n;
                acc_zero(n);
                #pragma unroll 1  // once per CTA: keep it small
                for (int t = 0; t < nt; ++t) acc_add_i64(n, (int64_t)hot[2 * S + t]);
                acc_to_cs(n, x.e, x.f);
            }
            break;
        }
    }
}

}  // namespace vr
