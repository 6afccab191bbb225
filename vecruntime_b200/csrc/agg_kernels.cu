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
#include <thrust/iterator/counting_iterator.h>

#include "agg_device.cuh"
#include "agg_kernels.cuh"

#include "agg_main.cuh"

namespace vr {

SmemMap smem_map(int stages, int stage_bytes, int tier_bytes) { return smem_map_impl(stages, stage_bytes, tier_bytes); }

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
        v.remap[c] = D.col_remap[c];
        v.remap_n[c] = D.col_remap_n[c];
    }
    v.sel = nullptr;
    uint32_t new_groups = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = (int64_t)blockIdx.x * blockDim.x;
    for (int64_t base = first; base < n; base += stride) {
        int64_t i = base + threadIdx.x;
        bool live[1] = {i < n};
        int64_t r[1] = {live[0] ? rows[i] : 0};
        hash_chunk<KW, 1>(P, D, v, r, live, 0, nullptr, 0, 0, g_probes, false, new_groups);
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
        case OP_SUM_I64:  // low word: signed (a sum of signed or unsigned 32-bit parts)
            wide_add_shifted(t, w[0], true, 0);
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
            wide_add_shifted(t, w[0], true, 0);
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

// Spark's decimal average: |s| (a 128-bit magnitude at the sum's scale) over
// a count, at a result scale `e` digits finer than the sum's: Decimal./
// (BigDecimal.divide(divisor, 39, HALF_UP)) then setScale(rs, HALF_UP)
// (DecimalAvgResult, VectorAggregates.scala:405-430). The quotient
// q = |s| * 10^e / count is computed exactly (256 bits, remainder r); the
// first rounding, at scale 39 (k = 39 - rs digits past the result scale),
// can only move the second one when the fraction r / count lies within
// 0.5 * 10^-k below one half: up <=> 10^k * (count - 2r) <= count, which for
// k >= 20 needs 10^k <= count < 2^64 and so reduces to 2r >= count.
// Returns false when the quotient leaves 128 bits (past any precision).
VR_DEV bool dec_avg_magnitude(uint64_t lo, uint64_t hi, uint64_t count, int e, int k, uint64_t& qlo, uint64_t& qhi) {
    uint64_t u[4] = {lo, hi, 0, 0};
    for (int i = 0; i < e; ++i) {  // * 10^e, e <= 38
        uint64_t carry = 0;
        for (int j = 0; j < 4; ++j) {
            const unsigned __int128 p = (unsigned __int128)u[j] * 10u + carry;
            u[j] = (uint64_t)p;
            carry = (uint64_t)(p >> 64);
        }
        if (carry) return false;
    }
    unsigned __int128 rem = 0;
    for (int j = 3; j >= 0; --j) {  // / count, word by word
        const unsigned __int128 cur = (rem << 64) | u[j];
        u[j] = (uint64_t)(cur / count);
        rem = cur % count;
    }
    const uint64_t r = (uint64_t)rem;
    bool up = r >= count - r;  // 2r >= count
    if (!up && k < 20) {
        unsigned __int128 p10 = 1;
        for (int i = 0; i < k; ++i) p10 *= 10u;
        up = p10 * (unsigned __int128)(count - 2 * r) <= (unsigned __int128)count;
    }
    if (up) {
        for (int j = 0; j < 4; ++j)
            if (++u[j] != 0) break;
    }
    if (u[2] | u[3]) return false;
    qlo = u[0];
    qhi = u[1];
    return true;
}

struct OutVal {
    uint64_t lo, hi;
    bool valid;
};

VR_DEV void emit_error(uint64_t* ctrl, int status) {
    atomicCAS((unsigned long long*)&ctrl[CTRL_EMIT_ERROR], 0ull, (unsigned long long)status);
}
// The first error of an emission together with the offending value (a
// decimal past its result type's precision), for Spark's message
// (NUMERIC_VALUE_OUT_OF_RANGE names the value): the thread that sets the
// status records it.
VR_DEV void emit_error_value(uint64_t* ctrl, int status, uint64_t lo, uint64_t hi, int precision, int scale) {
    if (atomicCAS((unsigned long long*)&ctrl[CTRL_EMIT_ERROR], 0ull, (unsigned long long)status) == 0ull) {
        ctrl[CTRL_EMIT_VALUE_LO] = lo;
        ctrl[CTRL_EMIT_VALUE_HI] = hi;
        ctrl[CTRL_EMIT_VALUE_TYPE] = ((uint64_t)(uint32_t)precision << 32) | (uint32_t)scale | (1ull << 63);
    }
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
            r.lo = (od.flags & OUTF_NULLCOUNT) ? acc[0] - acc[od.w0] : acc[od.w0];
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
            uint64_t cnt = (od.flags & OUTF_NULLCOUNT) ? acc[0] - acc[od.w1] : acc[od.w1];
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
                if ((od.flags & OUTF_FINAL) && !(od.flags & OUTF_NULL_ON_OVERFLOW)) {
                    if (!of && wide_fits_i128(t))
                        emit_error_value(ctrl, VR_ERR_DECIMAL_PRECISION, t.l[0], t.l[1], od.precision, od.scale);
                    else
                        emit_error(ctrl, VR_ERR_DECIMAL_PRECISION);
                }
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
                r.lo = ((od.flags & OUTF_NULLCOUNT) ? acc[0] - acc[od.w1] : acc[od.w1]) == 0 ? 1 : 0;
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
                    emit_error_value(ctrl, VR_ERR_DECIMAL_PRECISION, t.l[0], t.l[1], od.precision, od.scale);
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
        case OUT_AVG_DOUBLE: {
            // Average's evaluateExpression: sum / count as doubles, null when
            // no row counted (VectorAggregates.scala:1061-1064)
            uint64_t cnt;
            if (od.src_op == OP_SUM_I64) {
                bool of;
                cnt = op_total(OP_SUM_I64, acc + od.w1, of).l[0];
            } else {
                cnt = acc[od.w1];
            }
            if ((int64_t)cnt == 0) {
                r.valid = false;
                break;
            }
            r.lo = (uint64_t)__double_as_longlong(f64_total(acc + od.w0) / (double)(int64_t)cnt);
            break;
        }
        case OUT_DEC_AVG: {
            // If(count = 0, null, DecimalDivideWithOverflowCheck(sum, count, result type))
            bool of = false, sum_null;
            uint64_t cnt;
            Wide t;
            if (od.src_op == OP_MERGE_DAVG) {
                t = op_total(OP_MERGE_DAVG, acc + od.w0, of);
                cnt = op_total(OP_SUM_I64, acc + od.w1, of).l[0];
                sum_null = (acc[od.w0 + 6] & kFlagOverflow) != 0;
            } else {
                cnt = (od.flags & OUTF_NULLCOUNT) ? acc[0] - acc[od.w1] : acc[od.w1];
                if (od.src_op == OP_SUM_PROD && (acc[od.w0 + 6] & 1)) emit_error(ctrl, VR_ERR_DECIMAL_PRECISION);
                t = op_total(od.src_op, acc + od.w0, of);
                sum_null = of;
            }
            if ((int64_t)cnt == 0) {
                r.valid = false;
                break;
            }
            // the buffer's sum: null once it overflowed or past its precision
            sum_null = sum_null || !wide_fits_i128(t) ||
                       (!(od.flags & OUTF_UNGROUPED) && !within_precision(t.l[0], (int64_t)t.l[1], od.src_precision));
            if (sum_null) {
                r.valid = false;
                if (!(od.flags & OUTF_NULL_ON_OVERFLOW)) emit_error(ctrl, VR_ERR_DECIMAL_OVERFLOW);
                break;
            }
            const bool neg = (int64_t)t.l[1] < 0;
            uint64_t mlo = t.l[0], mhi = t.l[1];
            if (neg) {  // magnitude
                mlo = ~mlo + 1;
                mhi = ~mhi + (mlo == 0 ? 1 : 0);
            }
            uint64_t qlo, qhi;
            const bool q128 = dec_avg_magnitude(mlo, mhi, cnt, od.scale - od.src_scale, 39 - od.scale, qlo, qhi) &&
                              (int64_t)qhi >= 0;
            if (q128 && neg) {
                qlo = ~qlo + 1;
                qhi = ~qhi + (qlo == 0 ? 1 : 0);
            }
            if (!q128 || !within_precision(qlo, (int64_t)qhi, od.precision)) {
                // past the result precision: null, or NUMERIC_VALUE_OUT_OF_RANGE (ANSI)
                r.valid = false;
                if (!(od.flags & OUTF_NULL_ON_OVERFLOW)) {
                    if (q128)
                        emit_error_value(ctrl, VR_ERR_DECIMAL_PRECISION, qlo, qhi, od.precision, od.scale);
                    else
                        emit_error(ctrl, VR_ERR_DECIMAL_PRECISION);
                }
                break;
            }
            r.lo = qlo;
            r.hi = qhi;
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

// HashKernels.hashBytes (HashKernels.java:183-197): 4-byte little-endian
// words, then the tail bytes xor the length.
VR_DEV uint32_t jhash_bytes(const uint8_t* p, int32_t len) {
    uint32_t h = 0x1B873593u;
    int32_t i = 0;
    for (; i + 4 <= len; i += 4)
        h = jmix32(h, (uint32_t)p[i] | ((uint32_t)p[i + 1] << 8) | ((uint32_t)p[i + 2] << 16) | ((uint32_t)p[i + 3] << 24));
    uint32_t tail = 0;
    for (int shift = 0; i < len; ++i, shift += 8) tail |= (uint32_t)p[i] << shift;
    return jmix32(h, tail ^ (uint32_t)len);
}

constexpr uint32_t kNullMark = 0x7F4A7C15u;  // HashKernels.NULL_MARK

__global__ void k_hash_dictionary(vr_dictionary d, uint32_t* __restrict__ out) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < d.size; k += (int64_t)gridDim.x * blockDim.x) {
        const bool valid = d.validity == nullptr || ((d.validity[k >> 3] >> (k & 7)) & 1);
        out[k] = valid ? jhash_bytes(d.data + d.offsets[k], d.offsets[k + 1] - d.offsets[k]) : kNullMark;
    }
}

__global__ void k_hash_rows(int nk, const HashKey* __restrict__ keys, int64_t n, uint32_t* __restrict__ out,
                            int finish, uint32_t* bad_id) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t h = 0x2545F491u;
        for (int c = 0; c < nk; ++c) {
            const HashKey& col = keys[c];
            bool valid = col.validity == nullptr || ((col.validity[i >> 3] >> (i & 7)) & 1);
            uint32_t v;
            if (!valid) {
                v = kNullMark;
            } else {
                switch (col.lane) {
                    case VR_INT32:
                        v = (uint32_t) reinterpret_cast<const int32_t*>(col.data)[i];
                        break;
                    case VR_DICT32: {
                        const int32_t id = reinterpret_cast<const int32_t*>(col.data)[i];
                        if ((uint32_t)id < (uint32_t)col.dict_size) {
                            v = col.dict_hashes[id];
                        } else {
                            v = 0;
                            if (bad_id) *bad_id = 1;
                        }
                        break;
                    }
                    case VR_UTF8: {
                        const int32_t o = col.offsets[i];
                        v = jhash_bytes(reinterpret_cast<const uint8_t*>(col.data) + o, col.offsets[i + 1] - o);
                        break;
                    }
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
// The prebuilt aggregate kernels live in agg_aot_*.cu (one file per variant
// so they compile in parallel). The direct tier never packs keys: one
// variant serves every key width.
int aggregate_kernel_regs(int kw, int tier) {
    if (tier == kTierDirect) return aot_regs_direct();
    switch (kw) {
        case 1: return aot_regs_hash1();
        case 2: return aot_regs_hash2();
        case 3: return aot_regs_hash3();
        case 4: return aot_regs_hash4();
    }
    return 0;
}

cudaError_t launch_aggregate(int kw, int tier, const BatchDesc* descs, const LaunchCfg& cfg, int blocks,
                             uint64_t* tile_counter, cudaStream_t stream) {
    if (tier == kTierDirect) return aot_launch_direct(descs, cfg, blocks, tile_counter, stream);
    switch (kw) {
        case 1: return aot_launch_hash1(descs, cfg, blocks, tile_counter, stream);
        case 2: return aot_launch_hash2(descs, cfg, blocks, tile_counter, stream);
        case 3: return aot_launch_hash3(descs, cfg, blocks, tile_counter, stream);
        case 4: return aot_launch_hash4(descs, cfg, blocks, tile_counter, stream);
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
    thrust::counting_iterator<int64_t> it(0);
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

cudaError_t launch_hash_rows(int num_keys, const HashKey* keys_dev, int64_t n, uint32_t* out, int finish,
                             uint32_t* bad_id, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    k_hash_rows<<<grid_for(n, 256), 256, 0, stream>>>(num_keys, keys_dev, n, out, finish, bad_id);
    return cudaGetLastError();
}

cudaError_t launch_hash_dictionary(const vr_dictionary& dict, uint32_t* out, cudaStream_t stream) {
    if (dict.size <= 0) return cudaSuccess;
    k_hash_dictionary<<<grid_for(dict.size, 256), 256, 0, stream>>>(dict, out);
    return cudaGetLastError();
}

// Fixed device scratch for vr_hash_rows_noalloc: the key-column descriptors
// of one call, so that entry point never has to allocate the small table the
// kernel reads. One copy per device, shared by
// every call on that device. Nothing here needs to start at zero: each call
// writes the descriptors it uses before its kernel reads them.
static __device__ __align__(256) unsigned char g_hash_rows_scratch[kHashRowsScratchBytes];

cudaError_t hash_rows_scratch_address(void** out) {
    return cudaGetSymbolAddress(out, g_hash_rows_scratch);
}

}  // namespace vr
