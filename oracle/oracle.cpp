// CPU restatement of the reference's grouped aggregate (see oracle.h).
// TEST INFRASTRUCTURE ONLY -- the parity checker and the timed CPU baseline.
//
// Table: GroupKeyTable's general path (GroupKeyTable.java:709-764,
// 2296-2371, 2515-2561): row hash = HashKernels.init + mixColumn per key +
// finish; open addressing with linear probing over `hash & mask`; a slot holds
// (hash, group id); groups get dense ids in first-seen order and keep their
// key values per column (null as its own group, stored as 0 + null flag);
// 2048 initial slots, doubling when size * 10 > slots * 7 (rehash, :2631-2660).
// Accumulators: GroupedAccumulators.java, one accumulator per group, rows
// added sequentially in input order (the reference's strict mode, which is
// the default: spark.vecruntime.exec.strictFloatingPoint, VectorConf.scala:1080).
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

namespace {

typedef __int128 i128;
typedef unsigned __int128 u128;

thread_local std::string g_err;

// ---- HashKernels (HashKernels.java:36-64, 178-180; Decimal128.java:155-160)
const uint32_t SEED = 0x2545F491u;
const uint32_t MULT = 0x9E3779B1u;
const uint32_t NULL_MARK = 0x7F4A7C15u;

uint32_t mix32(uint32_t h, uint32_t v) {
    h = (h ^ v) * MULT;
    return h ^ (h >> 15);
}
uint32_t finish(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}
uint32_t fold(uint64_t v) { return (uint32_t)(v ^ (v >> 32)); }
// HashKernels.hashBytes (HashKernels.java:183-197): little-endian 4-byte
// words, then the remaining bytes packed low-first, xor the length.
uint32_t hash_bytes(const uint8_t* p, int32_t len) {
    uint32_t h = 0x1B873593u;
    int32_t i = 0;
    for (; i + 4 <= len; i += 4) {
        uint32_t w;
        std::memcpy(&w, p + i, 4);
        h = mix32(h, w);
    }
    uint32_t tail = 0;
    for (int shift = 0; i < len; ++i, shift += 8) tail |= (uint32_t)p[i] << shift;
    return mix32(h, tail ^ (uint32_t)len);
}
uint64_t dec_hash(uint64_t hi, uint64_t lo) {
    uint64_t h = lo * 0x9E3779B97F4A7C15ull;
    h ^= (h >> 32) ^ (hi * 0xC2B2AE3D27D4EB4Full);
    h ^= h >> 29;
    return h;
}

bool bit(const uint8_t* bm, int64_t i) { return (bm[i >> 3] >> (i & 7)) & 1; }
void set_bit(uint8_t* bm, int64_t i, bool v) {
    if (v)
        bm[i >> 3] |= (uint8_t)(1u << (i & 7));
    else
        bm[i >> 3] &= (uint8_t) ~(1u << (i & 7));
}

// ---- Decimal128 helpers (Decimal128.java:146-150: signed hi, unsigned lo)
i128 pow10_128(int p) {
    i128 v = 1;
    for (int i = 0; i < p; ++i) v *= 10;
    return v;
}
i128 abs128(i128 v) { return v < 0 ? -v : v; }

// A key value of one column: raw 64-bit words + null flag.
struct KeyVal {
    uint64_t lo = 0, hi = 0;
    bool null = false;
    bool operator==(const KeyVal& o) const { return null == o.null && lo == o.lo && hi == o.hi; }
};

enum { K_I64 = 0 };

// Per-function running state (one per group).
struct FnState {
    // counts / long sums
    int64_t count = 0;     // valid inputs (or rows for count(*))
    int64_t lsum = 0;      // LongSum running sum (wraps, or checked per row)
    double dsum = 0.0;     // DoubleSum strict running sum
    double csum = 0.0;     // Neumaier sum
    double ccomp = 0.0;    // Neumaier compensation
    int64_t lbest = 0;     // LongMinMax
    double dbest = 0.0;    // DoubleMinMax
    i128 wbest = 0;        // Decimal128MinMax
    bool any = false;
    i128 wide = 0;         // WideLongSum (hi, lo) as a signed 128-bit value
    bool overflowed = false;
    bool non_empty = false;  // merges
    int64_t count2 = 0;      // merges: second buffer's sum (counts)
};

struct Out {
    int kind, lane, precision, scale;
    int fn;  // function index
    int slot;
};

}  // namespace

struct orc_agg {
    vr_agg_spec spec{};
    std::vector<vr_column_type> cols;
    std::vector<int32_t> keys;
    std::vector<vr_agg_fn> fns;
    // table
    std::vector<int64_t> slots;  // (hash << 32) | gid, or -1
    int64_t mask = 0;
    std::vector<uint32_t> ghash;
    std::vector<std::vector<KeyVal>> kvals;  // [key][gid]
    std::vector<int64_t> rows;               // count(*) per group
    std::vector<std::vector<FnState>> st;    // [fn][gid]
    int64_t size = 0;
    int status = VR_OK;
    std::vector<vr_column_type> out_types;
    // VR_COL_BATCH_DICTIONARY keys: the table dictionary (strings -> ids in
    // first-use order, GroupKeyTable.toIds, GroupKeyTable.java:1308-1430)
    std::vector<std::map<std::string, int32_t>> dict_ids;  // [key]
    std::vector<std::vector<std::string>> dict_strings;   // [key][id]
};

namespace {

int fail(orc_agg* a, int code, const char* msg) {
    g_err = msg;
    if (a && a->status == VR_OK) a->status = code;
    return code;
}

KeyVal key_at(const vr_column_type& t, const vr_column& c, int64_t i) {
    KeyVal k;
    if (c.validity && !bit(c.validity, i)) {
        k.null = true;
        return k;
    }
    switch (t.lane) {
        case VR_INT32:
        case VR_DICT32: k.lo = (uint64_t)(uint32_t)((const int32_t*)c.data)[i]; break;
        case VR_INT64:
        case VR_FLOAT64: k.lo = ((const uint64_t*)c.data)[i]; break;
        case VR_BOOL: k.lo = bit((const uint8_t*)c.data, i) ? 1 : 0; break;
        case VR_DECIMAL128:
            k.lo = ((const uint64_t*)c.data)[2 * i];
            k.hi = ((const uint64_t*)c.data)[2 * i + 1];
            break;
    }
    return k;
}

uint32_t key_hash_value(int lane, const KeyVal& k) {
    if (k.null) return NULL_MARK;
    switch (lane) {
        case VR_INT32:
        case VR_DICT32:
        case VR_BOOL: return (uint32_t)k.lo;
        case VR_INT64:
        case VR_FLOAT64: return fold(k.lo);
        case VR_DECIMAL128: return fold(dec_hash(k.hi, k.lo));
    }
    return 0;
}

void rehash(orc_agg* a) {
    int64_t n = (int64_t)a->slots.size() * 2;
    std::vector<int64_t> ns(n, -1);
    int64_t m = n - 1;
    for (int64_t g = 0; g < a->size; ++g) {
        int64_t pos = a->ghash[g] & m;
        while (ns[pos] != -1) pos = (pos + 1) & m;
        ns[pos] = ((int64_t)a->ghash[g] << 32) | g;
    }
    a->slots.swap(ns);
    a->mask = m;
}

int64_t new_group(orc_agg* a, uint32_t hash, const std::vector<KeyVal>& key) {
    int64_t g = a->size++;
    a->ghash.push_back(hash);
    for (size_t k = 0; k < key.size(); ++k) a->kvals[k].push_back(key[k]);
    a->rows.push_back(0);
    for (auto& v : a->st) v.emplace_back();
    return g;
}

// lookupOrInsert (GroupKeyTable.java:2296-2323): probe, compare hash then keys.
int64_t lookup_or_insert(orc_agg* a, uint32_t hash, const std::vector<KeyVal>& key) {
    int64_t pos = hash & a->mask;
    while (true) {
        int64_t e = a->slots[pos];
        if (e == -1) {
            int64_t g = new_group(a, hash, key);
            a->slots[pos] = ((int64_t)hash << 32) | g;
            if (a->size * 10 > (int64_t)a->slots.size() * 7) rehash(a);
            return g;
        }
        int64_t g = e & 0xffffffffll;
        if ((uint32_t)(e >> 32) == hash) {
            bool eq = true;
            for (size_t k = 0; k < key.size() && eq; ++k) eq = a->kvals[k][g] == key[k];
            if (eq) return g;
        }
        pos = (pos + 1) & a->mask;
    }
}

bool valid(const vr_column& c, int64_t i) { return !c.validity || bit(c.validity, i); }
int64_t ld_int(const vr_column_type& t, const vr_column& c, int64_t i) {
    return (t.lane == VR_INT32 || t.lane == VR_DICT32) ? (int64_t)((const int32_t*)c.data)[i] : ((const int64_t*)c.data)[i];
}
double ld_f64(const vr_column& c, int64_t i) { return ((const double*)c.data)[i]; }
i128 ld_d128(const vr_column& c, int64_t i) {
    const uint64_t* p = (const uint64_t*)c.data + 2 * i;
    return (i128)(((u128)p[1] << 64) | p[0]);
}

// CompareOp.nanSafeCompare (CompareOp.java:68-81)
int nan_safe_compare(double x, double y) {
    bool xn = std::isnan(x), yn = std::isnan(y);
    if ((xn && yn) || x == y) return 0;
    if (xn) return 1;
    if (yn) return -1;
    return x > y ? 1 : -1;
}

void neumaier(FnState& s, double x) {
    double t = s.csum + x;
    if (std::fabs(s.csum) >= std::fabs(x))
        s.ccomp += (s.csum - t) + x;
    else
        s.ccomp += (x - t) + s.csum;
    s.csum = t;
}

// WideLongSum.addWide (GroupedAccumulators.java:768-782): signed 128-bit add,
// sticky overflow when the running total leaves 128 bits.
void add_wide(FnState& s, i128 x) {
    u128 r = (u128)s.wide + (u128)x;
    i128 ri = (i128)r;
    if (((s.wide ^ ri) & (x ^ ri)) < 0) s.overflowed = true;
    s.wide = ri;
}

// The exact product of a fused decimal product, or false when it is null
// (past 128 bits or past its declared precision: Spark's CheckOverflow).
bool product(const orc_agg* a, const vr_agg_fn& f, const vr_batch& b, int64_t i, i128& out, bool& null_row) {
    null_row = false;
    i128 p = 1;
    for (int t = 0; t < f.num_terms; ++t) {
        const vr_column& c = b.columns[f.terms[t].column];
        if (!valid(c, i)) {
            null_row = true;
            return true;
        }
        int64_t v = ((const int64_t*)c.data)[i];
        i128 term = (i128)f.terms[t].addend + (f.terms[t].sign < 0 ? -(i128)v : (i128)v);
        i128 q;
        if (__builtin_mul_overflow(p, term, &q)) return false;
        p = q;
    }
    int prec = f.product_precision > 0 ? std::min(38, f.product_precision) : 38;
    if (abs128(p) >= pow10_128(prec)) return false;
    out = p;
    (void)a;
    return true;
}

int update_row(orc_agg* a, const vr_batch& b, int64_t i, int64_t g) {
    a->rows[g]++;
    for (size_t fi = 0; fi < a->fns.size(); ++fi) {
        const vr_agg_fn& f = a->fns[fi];
        FnState& s = a->st[fi][g];
        const vr_column* in = f.input >= 0 ? &b.columns[f.input] : nullptr;
        const vr_column_type* it = f.input >= 0 ? &a->cols[f.input] : nullptr;
        switch (f.kind) {
            case VR_FN_COUNT_STAR: s.count++; break;
            case VR_FN_COUNT:
                if (valid(*in, i)) s.count++;
                break;
            case VR_FN_SUM_LONG: {  // LongSum (GroupedAccumulators.java:363-624)
                if (!valid(*in, i)) break;
                int64_t x = ld_int(*it, *in, i);
                if (f.flags & VR_FN_CHECKED) {
                    int64_t r;
                    if (__builtin_add_overflow(s.lsum, x, &r)) return fail(a, VR_ERR_OVERFLOW, "long overflow");
                    s.lsum = r;
                } else {
                    s.lsum = (int64_t)((uint64_t)s.lsum + (uint64_t)x);
                }
                s.count++;
                break;
            }
            case VR_FN_SUM_DOUBLE:
            case VR_FN_AVG_DOUBLE: {  // DoubleSum strict (GroupedAccumulators.java:232-241)
                if (!valid(*in, i)) break;
                double x = ld_f64(*in, i);
                s.dsum += x;
                neumaier(s, x);
                s.count++;
                break;
            }
            case VR_FN_MIN:
            case VR_FN_MAX: {  // LongMinMax / DoubleMinMax / Decimal128MinMax offer() (:1248-1258, :1327-1334, :1410-1422)
                if (!valid(*in, i)) break;
                bool mn = f.kind == VR_FN_MIN;
                s.count++;
                if (it->lane == VR_FLOAT64) {
                    double x = ld_f64(*in, i);
                    if (!s.any) {
                        s.dbest = x;
                        s.any = true;
                    } else {
                        int c = nan_safe_compare(x, s.dbest);
                        if (mn ? c < 0 : c > 0) s.dbest = x;
                    }
                } else if (it->lane == VR_DECIMAL128) {
                    i128 x = ld_d128(*in, i);
                    if (!s.any || (mn ? x < s.wbest : x > s.wbest)) s.wbest = x;
                    s.any = true;
                } else {
                    int64_t x = ld_int(*it, *in, i);
                    if (!s.any || (mn ? x < s.lbest : x > s.lbest)) s.lbest = x;
                    s.any = true;
                }
                break;
            }
            case VR_FN_SUM_DECIMAL:
            case VR_FN_AVG_DECIMAL: {  // WideLongSum.add / addWide (GroupedAccumulators.java:768-824)
                if (f.num_terms > 0) {
                    i128 p;
                    bool null_row;
                    if (!product(a, f, b, i, p, null_row)) {
                        if (f.flags & VR_FN_CHECKED)
                            return fail(a, VR_ERR_DECIMAL_PRECISION, "decimal product past its precision");
                        break;  // the product is null for this row
                    }
                    if (null_row) break;
                    add_wide(s, p);
                    s.count++;
                    break;
                }
                if (!valid(*in, i)) break;
                if (it->lane == VR_DECIMAL128)
                    add_wide(s, ld_d128(*in, i));
                else
                    s.wide += (i128)ld_int(*it, *in, i);  // INT64 lane: add(), no overflow flag
                s.count++;
                break;
            }
            case VR_FN_COUNT_MERGE:  // CountMergeAgg: LongSum over the counts (unchecked)
                if (valid(*in, i)) s.lsum = (int64_t)((uint64_t)s.lsum + (uint64_t)ld_int(*it, *in, i));
                break;
            case VR_FN_AVG_DOUBLE_MERGE: {  // AverageMergeAgg: DoubleSum(sum) + LongSum(count)
                const vr_column& cc = b.columns[f.input2];
                if (valid(*in, i)) {
                    double x = ld_f64(*in, i);
                    s.dsum += x;
                    neumaier(s, x);
                }
                if (valid(cc, i)) s.count2 = (int64_t)((uint64_t)s.count2 + (uint64_t)((const int64_t*)cc.data)[i]);
                break;
            }
            case VR_FN_SUM_DECIMAL_MERGE: {  // WideDecimalSumMergeAgg.State.merge (VectorAggregates.scala:705-724)
                const vr_column& ec = b.columns[f.input2];
                if (!valid(ec, i) || bit((const uint8_t*)ec.data, i)) break;
                s.non_empty = true;
                if (!valid(*in, i)) {
                    s.overflowed = true;
                } else if (!s.overflowed) {
                    i128 x = ld_d128(*in, i);
                    u128 r = (u128)s.wide + (u128)x;
                    i128 ri = (i128)r;
                    if (((s.wide ^ ri) & (x ^ ri)) < 0)
                        s.overflowed = true;
                    else
                        s.wide = ri;
                }
                break;
            }
            case VR_FN_AVG_DECIMAL_MERGE: {  // WideDecimalAvgMergeAgg.State.merge (VectorAggregates.scala:557-590)
                const vr_column& cc = b.columns[f.input2];
                if (valid(cc, i)) s.count2 += ((const int64_t*)cc.data)[i];
                if (!valid(*in, i)) {
                    s.overflowed = true;
                } else if (!s.overflowed) {
                    i128 x = ld_d128(*in, i);
                    u128 r = (u128)s.wide + (u128)x;
                    i128 ri = (i128)r;
                    if (((s.wide ^ ri) & (x ^ ri)) < 0)
                        s.overflowed = true;
                    else
                        s.wide = ri;
                }
                break;
            }
            default:
                return fail(a, VR_ERR_UNSUPPORTED, "function kind");
        }
    }
    return VR_OK;
}

void add_out(orc_agg* a, int lane, int precision, int scale) {
    vr_column_type t;
    std::memset(&t, 0, sizeof(t));
    t.lane = lane;
    t.precision = precision;
    t.scale = scale;
    t.nullable = 1;
    a->out_types.push_back(t);
}

// Output schema: keys, then each function's Spark buffer slots
// (VectorAggFunction.bufferTypes, VectorAggregates.scala).
// A decimal average's result type: given, or Spark's Decimal(p + 4, s + 4)
// of the input behind the Decimal(p + 10, s) buffer, bounded to 38.
bool avg_result_type(const vr_agg_fn& f, int& rp, int& rs) {
    if (f.result_precision > 0) {
        rp = f.result_precision;
        rs = f.result_scale;
    } else {
        if (f.precision >= 38) return false;
        rp = std::min(f.precision - 6, 38);
        rs = std::min(f.scale + 4, 38);
    }
    return rp >= 1 && rp <= 38 && rs >= f.scale && rs <= rp;
}

// Unsigned 256-bit integer for the average's division.
struct U256 {
    uint64_t w[4] = {0, 0, 0, 0};
};
bool u256_mul_small(U256& a, uint64_t m) {
    u128 carry = 0;
    for (int i = 0; i < 4; ++i) {
        u128 p = (u128)a.w[i] * m + carry;
        a.w[i] = (uint64_t)p;
        carry = p >> 64;
    }
    return carry == 0;
}
void u256_add_small(U256& a, uint64_t v) {
    u128 carry = v;
    for (int i = 0; i < 4 && carry; ++i) {
        u128 s = (u128)a.w[i] + carry;
        a.w[i] = (uint64_t)s;
        carry = s >> 64;
    }
}
uint64_t u256_divmod_small(U256& a, uint64_t d) {
    u128 rem = 0;
    for (int i = 3; i >= 0; --i) {
        u128 cur = (rem << 64) | a.w[i];
        a.w[i] = (uint64_t)(cur / d);
        rem = cur % d;
    }
    return (uint64_t)rem;
}

// Spark's Decimal./ as DecimalAvgResult evaluates it: BigDecimal(sum, ss)
// .divide(BigDecimal(count), 39, HALF_UP).setScale(rs, HALF_UP), literally
// in two roundings (VectorAggregates.scala:405-430). False when the result
// reaches 10^rp.
bool spark_decimal_avg(i128 sum, int64_t count, int ss, int rs, int rp, i128& out) {
    const bool neg = sum < 0;
    u128 mag = neg ? (u128)0 - (u128)sum : (u128)sum;
    U256 n;
    n.w[0] = (uint64_t)mag;
    n.w[1] = (uint64_t)(mag >> 64);
    for (int i = 0; i < 39 - ss; ++i)
        if (!u256_mul_small(n, 10)) return false;
    const uint64_t r = u256_divmod_small(n, (uint64_t)count);  // the quotient at scale 39
    if (2 * (u128)r >= (u128)count) u256_add_small(n, 1);
    const int m = 39 - rs;  // then to the result scale, half up
    if (m > 0) {
        U256 half;
        half.w[0] = 5;
        for (int i = 0; i < m - 1; ++i) u256_mul_small(half, 10);
        u128 carry = 0;
        for (int i = 0; i < 4; ++i) {
            u128 s = (u128)n.w[i] + half.w[i] + carry;
            n.w[i] = (uint64_t)s;
            carry = s >> 64;
        }
        for (int i = 0; i < m; ++i) u256_divmod_small(n, 10);
    }
    if (n.w[2] || n.w[3]) return false;
    u128 q = ((u128)n.w[1] << 64) | n.w[0];
    if (q >= (u128)pow10_128(rp)) return false;
    out = neg ? -(i128)q : (i128)q;
    return true;
}

int build_outputs(orc_agg* a) {
    for (int32_t k : a->keys) {
        const vr_column_type& t = a->cols[k];
        add_out(a, t.lane, t.lane == VR_DECIMAL128 || t.precision > 0 ? t.precision : 0, t.scale);
    }
    for (auto& f : a->fns) {
        const vr_column_type* it = f.input >= 0 ? &a->cols[f.input] : nullptr;
        switch (f.kind) {
            case VR_FN_COUNT_STAR:
            case VR_FN_COUNT:
            case VR_FN_SUM_LONG:
            case VR_FN_COUNT_MERGE: add_out(a, VR_INT64, 0, 0); break;
            case VR_FN_SUM_DOUBLE: add_out(a, VR_FLOAT64, 0, 0); break;
            case VR_FN_AVG_DOUBLE:
            case VR_FN_AVG_DOUBLE_MERGE:
                add_out(a, VR_FLOAT64, 0, 0);
                add_out(a, VR_INT64, 0, 0);
                break;
            case VR_FN_MIN:
            case VR_FN_MAX: add_out(a, it->lane, it->precision, it->scale); break;
            case VR_FN_SUM_DECIMAL:
            case VR_FN_SUM_DECIMAL_MERGE:
                add_out(a, VR_DECIMAL128, f.precision, f.scale);
                add_out(a, VR_BOOL, 0, 0);
                break;
            case VR_FN_AVG_DECIMAL:
            case VR_FN_AVG_DECIMAL_MERGE:
                if (f.flags & VR_FN_FINAL) {  // the result type: an INT64 lane up to 18 digits
                    int rp, rs;
                    if (!avg_result_type(f, rp, rs)) return fail(a, VR_ERR_INVALID, "decimal average result type");
                    add_out(a, rp <= 18 ? VR_INT64 : VR_DECIMAL128, rp, rs);
                } else {
                    add_out(a, VR_DECIMAL128, f.precision, f.scale);
                }
                add_out(a, VR_INT64, 0, 0);
                break;
            default: return fail(a, VR_ERR_UNSUPPORTED, "function kind");
        }
    }
    return VR_OK;
}

struct Cell {
    bool valid = true;
    uint64_t lo = 0, hi = 0;
};

void put(const vr_out_column& o, int lane, int64_t row, const Cell& c) {
    if (o.validity) set_bit(o.validity, row, c.valid);
    switch (lane) {
        case VR_INT32:
        case VR_DICT32: ((int32_t*)o.data)[row] = c.valid ? (int32_t)c.lo : 0; break;
        case VR_INT64:
        case VR_FLOAT64: ((uint64_t*)o.data)[row] = c.valid ? c.lo : 0; break;
        case VR_BOOL: set_bit((uint8_t*)o.data, row, c.valid && c.lo != 0); break;
        case VR_DECIMAL128:
            ((uint64_t*)o.data)[2 * row] = c.valid ? c.lo : 0;
            ((uint64_t*)o.data)[2 * row + 1] = c.valid ? c.hi : 0;
            break;
    }
}

Cell dec_cell(i128 v) {
    Cell c;
    c.lo = (uint64_t)(u128)v;
    c.hi = (uint64_t)((u128)v >> 64);
    return c;
}
Cell f64_cell(double d) {
    Cell c;
    std::memcpy(&c.lo, &d, 8);
    return c;
}
Cell null_cell() {
    Cell c;
    c.valid = false;
    return c;
}

// One decimal average result: If(count = 0, null, DecimalDivideWithOverflowCheck(
// sum, count, result type)): a null sum is null or ARITHMETIC_OVERFLOW (ANSI),
// a result past its precision null or NUMERIC_VALUE_OUT_OF_RANGE (ANSI).
int put_avg(orc_agg* a, const vr_out_column& out, int64_t o, const vr_agg_fn& f, int64_t count, bool sum_null,
            i128 sum) {
    int rp, rs;
    avg_result_type(f, rp, rs);
    const int lane = rp <= 18 ? VR_INT64 : VR_DECIMAL128;
    const bool nullov = (f.flags & VR_FN_NULL_ON_OVERFLOW) != 0;
    if (count == 0) {
        put(out, lane, o, null_cell());
        return VR_OK;
    }
    if (sum_null) {
        if (!nullov) return fail(a, VR_ERR_DECIMAL_OVERFLOW, "overflow in sum of decimals");
        put(out, lane, o, null_cell());
        return VR_OK;
    }
    i128 q;
    if (!spark_decimal_avg(sum, count, f.scale, rs, rp, q)) {
        if (!nullov) return fail(a, VR_ERR_DECIMAL_PRECISION, "decimal precision");
        put(out, lane, o, null_cell());
        return VR_OK;
    }
    Cell c = dec_cell(q);
    put(out, lane, o, c);
    return VR_OK;
}

}  // namespace

extern "C" {

int orc_agg_create(const vr_agg_spec* spec, orc_agg** out) {
    if (!spec || !out) return VR_ERR_INVALID;
    orc_agg* a = new orc_agg();
    a->cols.assign(spec->columns, spec->columns + spec->num_columns);
    a->keys.assign(spec->key_columns, spec->key_columns + spec->num_keys);
    a->fns.assign(spec->fns, spec->fns + spec->num_fns);
    a->spec = *spec;
    a->spec.columns = a->cols.data();
    a->spec.key_columns = a->keys.data();
    a->spec.fns = a->fns.data();
    a->slots.assign(2048, -1);  // INITIAL_CAPACITY * 2 (GroupKeyTable.java:574)
    a->mask = 2047;
    a->kvals.resize(a->keys.size());
    a->dict_ids.resize(a->keys.size());
    a->dict_strings.resize(a->keys.size());
    a->st.resize(a->fns.size());
    int rc = build_outputs(a);
    if (rc != VR_OK) {
        delete a;
        return rc;
    }
    *out = a;
    return VR_OK;
}

// Key k of row i; a key whose batches bring dictionaries becomes the table
// id of its string (a null entry: a null key).
KeyVal key_of(orc_agg* a, size_t k, const vr_batch& b, int64_t i) {
    const vr_column_type& t = a->cols[a->keys[k]];
    const vr_column& col = b.columns[a->keys[k]];
    KeyVal kv = key_at(t, col, i);
    if (!(t.flags & VR_COL_BATCH_DICTIONARY) || kv.null) return kv;
    const vr_dictionary& d = *col.dictionary;
    const int32_t e = (int32_t)kv.lo;
    if (e < 0 || e >= d.size || (d.validity && !bit(d.validity, e))) {
        kv.null = true;  // an id past the dictionary is refused by update; a null entry is a null key
        kv.lo = 0;
        return kv;
    }
    std::string s((const char*)d.data + d.offsets[e], (size_t)(d.offsets[e + 1] - d.offsets[e]));
    auto& ids = a->dict_ids[k];
    auto it = ids.find(s);
    if (it == ids.end()) {
        it = ids.emplace(s, (int32_t)ids.size()).first;
        a->dict_strings[k].push_back(s);
    }
    kv.lo = (uint64_t)(uint32_t)it->second;
    return kv;
}

int orc_agg_update(orc_agg* a, const vr_batch* b, int64_t chunk) {
    if (!a || !b) return VR_ERR_INVALID;
    if (a->status != VR_OK) return a->status;
    for (size_t k = 0; k < a->keys.size(); ++k) {
        const vr_column_type& t = a->cols[a->keys[k]];
        if (!(t.flags & VR_COL_BATCH_DICTIONARY)) continue;
        const vr_column& col = b->columns[a->keys[k]];
        if (!col.dictionary) return fail(a, VR_ERR_INVALID, "a key declared with batch dictionaries came without one");
        for (int64_t i = 0; i < b->num_rows; ++i) {
            if (col.validity && !bit(col.validity, i)) continue;
            const int32_t e = ((const int32_t*)col.data)[i];
            if (e < 0 || e >= col.dictionary->size) return fail(a, VR_ERR_INVALID, "dictionary id outside its dictionary");
        }
    }
    const int64_t n = b->num_rows;
    if (chunk <= 0) chunk = n > 0 ? n : 1;
    std::vector<uint32_t> hashes((size_t)std::min(chunk, std::max<int64_t>(n, 1)));
    std::vector<KeyVal> key(a->keys.size());
    const size_t nk = a->keys.size();
    for (int64_t c0 = 0; c0 < n; c0 += chunk) {
        int64_t m = std::min(chunk, n - c0);
        // HashKernels.init + mixColumn per key column, then finish per row
        for (int64_t r = 0; r < m; ++r) hashes[r] = SEED;
        for (size_t k = 0; k < nk; ++k) {
            const vr_column_type& t = a->cols[a->keys[k]];
            const vr_column& col = b->columns[a->keys[k]];
            (void)col;
            for (int64_t r = 0; r < m; ++r) hashes[r] = mix32(hashes[r], key_hash_value(t.lane, key_of(a, k, *b, c0 + r)));
        }
        for (int64_t r = 0; r < m; ++r) {
            int64_t i = c0 + r;
            if (b->selection && !bit(b->selection, i)) continue;  // unselected rows create no group
            for (size_t k = 0; k < nk; ++k) key[k] = key_of(a, k, *b, i);
            int64_t g = nk == 0 ? (a->size == 0 ? new_group(a, 0, key) : 0) : lookup_or_insert(a, finish(hashes[r]), key);
            int rc = update_row(a, *b, i, g);
            if (rc != VR_OK) return rc;
        }
    }
    return VR_OK;
}

int64_t orc_agg_num_groups(const orc_agg* a) { return a ? a->size : -1; }
int orc_agg_num_outputs(const orc_agg* a) { return a ? (int)a->out_types.size() : -1; }
int orc_agg_output_type(const orc_agg* a, int i, vr_column_type* t) {
    if (!a || !t || i < 0 || i >= (int)a->out_types.size()) return VR_ERR_INVALID;
    *t = a->out_types[i];
    return VR_OK;
}

int orc_agg_emit(orc_agg* a, int64_t from, int64_t to, const vr_out_column* outs, int fp_mode) {
    if (!a || !outs || from < 0 || to < from || to > a->size) return VR_ERR_INVALID;
    if (a->status != VR_OK) return a->status;
    for (int64_t g = from; g < to; ++g) {
        int64_t o = g - from;
        int j = 0;
        for (size_t k = 0; k < a->keys.size(); ++k, ++j) {  // GroupKeyTable.writeKeys (:2851-2920)
            const KeyVal& kv = a->kvals[k][g];
            Cell c;
            c.valid = !kv.null;
            c.lo = kv.lo;
            c.hi = kv.hi;
            put(outs[j], a->out_types[j].lane, o, c);
        }
        for (size_t fi = 0; fi < a->fns.size(); ++fi) {
            const vr_agg_fn& f = a->fns[fi];
            const FnState& s = a->st[fi][g];
            bool comp = fp_mode == ORC_FP_COMPENSATED;
            double dval = comp ? s.csum + s.ccomp : s.dsum;
            bool final_ = (f.flags & VR_FN_FINAL) != 0;
            bool nullov = (f.flags & VR_FN_NULL_ON_OVERFLOW) != 0;
            switch (f.kind) {
                case VR_FN_COUNT_STAR:
                case VR_FN_COUNT: {
                    Cell c;
                    c.lo = (uint64_t)s.count;
                    put(outs[j], VR_INT64, o, c);
                    ++j;
                    break;
                }
                case VR_FN_SUM_LONG: {  // SumLongAgg.writeBuffer (VectorAggregates.scala:179-198)
                    Cell c = s.count == 0 ? null_cell() : Cell();
                    c.lo = (uint64_t)s.lsum;
                    put(outs[j], VR_INT64, o, c);
                    ++j;
                    break;
                }
                case VR_FN_SUM_DOUBLE:  // SumDoubleAgg: null until the first non-null input
                    put(outs[j], VR_FLOAT64, o, s.count == 0 ? null_cell() : f64_cell(dval));
                    ++j;
                    break;
                case VR_FN_AVG_DOUBLE: {  // AverageAgg: (sum, count), never null; Complete: sum / count
                    if (final_)
                        put(outs[j], VR_FLOAT64, o, s.count == 0 ? null_cell() : f64_cell(dval / (double)s.count));
                    else
                        put(outs[j], VR_FLOAT64, o, f64_cell(dval));
                    Cell c;
                    c.lo = (uint64_t)s.count;
                    put(outs[j + 1], VR_INT64, o, c);
                    j += 2;
                    break;
                }
                case VR_FN_MIN:
                case VR_FN_MAX: {
                    int lane = a->out_types[j].lane;
                    Cell c = s.any ? Cell() : null_cell();
                    if (lane == VR_FLOAT64)
                        c = s.any ? f64_cell(s.dbest) : null_cell();
                    else if (lane == VR_DECIMAL128)
                        c = s.any ? dec_cell(s.wbest) : null_cell();
                    else
                        c.lo = (uint64_t)s.lbest;
                    put(outs[j], lane, o, c);
                    ++j;
                    break;
                }
                case VR_FN_SUM_DECIMAL:
                case VR_FN_AVG_DECIMAL: {  // WideDecimalSumAgg / WideDecimalAvgAgg buffers (:329-347, :374-389, :466-477)
                    i128 limit = pow10_128(f.precision);
                    if (f.kind == VR_FN_AVG_DECIMAL && final_) {  // Complete: the average itself
                        int rc = put_avg(a, outs[j], o, f, s.count, s.overflowed || abs128(s.wide) >= limit, s.wide);
                        if (rc != VR_OK) return rc;
                        Cell c2;
                        c2.lo = (uint64_t)s.count;
                        put(outs[j + 1], VR_INT64, o, c2);
                        j += 2;
                        break;
                    }
                    bool past = s.overflowed || abs128(s.wide) >= limit;
                    Cell c;
                    if (s.count == 0) {
                        c = (final_ && f.kind == VR_FN_SUM_DECIMAL) ? null_cell() : dec_cell(0);
                    } else if (past) {
                        if (final_ && !nullov && f.kind == VR_FN_SUM_DECIMAL)
                            return fail(a, VR_ERR_DECIMAL_PRECISION, "decimal precision");
                        c = null_cell();
                    } else {
                        c = dec_cell(s.wide);
                    }
                    put(outs[j], VR_DECIMAL128, o, c);
                    Cell c2;
                    if (f.kind == VR_FN_SUM_DECIMAL) {
                        c2.lo = s.count == 0 ? 1 : 0;
                        put(outs[j + 1], VR_BOOL, o, c2);
                    } else {
                        c2.lo = (uint64_t)s.count;
                        put(outs[j + 1], VR_INT64, o, c2);
                    }
                    j += 2;
                    break;
                }
                case VR_FN_COUNT_MERGE: {
                    Cell c;
                    c.lo = (uint64_t)s.lsum;
                    put(outs[j], VR_INT64, o, c);
                    ++j;
                    break;
                }
                case VR_FN_AVG_DOUBLE_MERGE: {  // Final: sum / count, null for no rows
                    if (final_)
                        put(outs[j], VR_FLOAT64, o, s.count2 == 0 ? null_cell() : f64_cell(dval / (double)s.count2));
                    else
                        put(outs[j], VR_FLOAT64, o, f64_cell(dval));
                    Cell c;
                    c.lo = (uint64_t)s.count2;
                    put(outs[j + 1], VR_INT64, o, c);
                    j += 2;
                    break;
                }
                case VR_FN_SUM_DECIMAL_MERGE: {  // State.value / write (VectorAggregates.scala:727-766)
                    i128 limit = pow10_128(f.precision);
                    Cell c;
                    if (!s.non_empty) {
                        c = final_ ? null_cell() : dec_cell(0);
                    } else if (s.overflowed) {
                        if (final_ && !nullov) return fail(a, VR_ERR_DECIMAL_OVERFLOW, "overflow in sum of decimals");
                        c = null_cell();
                    } else if (abs128(s.wide) >= limit) {
                        if (final_ && !nullov) return fail(a, VR_ERR_DECIMAL_PRECISION, "decimal precision");
                        c = null_cell();
                    } else {
                        c = dec_cell(s.wide);
                    }
                    put(outs[j], VR_DECIMAL128, o, c);
                    Cell c2;
                    c2.lo = s.non_empty ? 0 : 1;
                    put(outs[j + 1], VR_BOOL, o, c2);
                    j += 2;
                    break;
                }
                case VR_FN_AVG_DECIMAL_MERGE: {  // State.sum (VectorAggregates.scala:600-603)
                    i128 limit = pow10_128(f.precision);
                    if (final_) {  // DecimalAvgResult; an ungrouped Final keeps a sum past the buffer precision
                        bool past = s.overflowed || (!a->keys.empty() && abs128(s.wide) >= limit);
                        int rc = put_avg(a, outs[j], o, f, s.count2, past, s.wide);
                        if (rc != VR_OK) return rc;
                    } else {
                        Cell c = (s.overflowed || abs128(s.wide) >= limit) ? null_cell() : dec_cell(s.wide);
                        put(outs[j], VR_DECIMAL128, o, c);
                    }
                    Cell c2;
                    c2.lo = (uint64_t)s.count2;
                    put(outs[j + 1], VR_INT64, o, c2);
                    j += 2;
                    break;
                }
            }
        }
    }
    return VR_OK;
}

int orc_agg_merge(orc_agg* dst, const orc_agg* src) {
    if (!dst || !src) return VR_ERR_INVALID;
    for (int64_t g = 0; g < src->size; ++g) {
        std::vector<KeyVal> key(src->keys.size());
        uint32_t h = src->ghash[g];
        bool rehash = false;
        for (size_t k = 0; k < key.size(); ++k) {
            key[k] = src->kvals[k][g];
            if ((src->cols[src->keys[k]].flags & VR_COL_BATCH_DICTIONARY) && !key[k].null) {
                // the source's table id -> its string -> this table's id
                const std::string& s = src->dict_strings[k][(size_t)key[k].lo];
                auto it = dst->dict_ids[k].find(s);
                if (it == dst->dict_ids[k].end()) {
                    it = dst->dict_ids[k].emplace(s, (int32_t)dst->dict_ids[k].size()).first;
                    dst->dict_strings[k].push_back(s);
                }
                key[k].lo = (uint64_t)(uint32_t)it->second;
                rehash = true;
            }
        }
        if (rehash) {
            h = SEED;
            for (size_t k = 0; k < key.size(); ++k) h = mix32(h, key_hash_value(src->cols[src->keys[k]].lane, key[k]));
            h = finish(h);
        }
        int64_t d = key.empty() ? (dst->size == 0 ? new_group(dst, 0, key) : 0) : lookup_or_insert(dst, h, key);
        dst->rows[d] += src->rows[g];
        for (size_t fi = 0; fi < dst->fns.size(); ++fi) {
            FnState& a = dst->st[fi][d];
            const FnState& b = src->st[fi][g];
            const vr_agg_fn& f = dst->fns[fi];
            a.count += b.count;
            a.count2 += b.count2;
            a.lsum = (int64_t)((uint64_t)a.lsum + (uint64_t)b.lsum);
            a.dsum += b.dsum;
            neumaier(a, b.csum);
            a.ccomp += b.ccomp;
            bool mn = f.kind == VR_FN_MIN;
            if (b.any) {
                if (!a.any) {
                    a.lbest = b.lbest;
                    a.dbest = b.dbest;
                    a.wbest = b.wbest;
                } else {
                    if (mn ? b.lbest < a.lbest : b.lbest > a.lbest) a.lbest = b.lbest;
                    int c = nan_safe_compare(b.dbest, a.dbest);
                    if (mn ? c < 0 : c > 0) a.dbest = b.dbest;
                    if (mn ? b.wbest < a.wbest : b.wbest > a.wbest) a.wbest = b.wbest;
                }
                a.any = true;
            }
            if (b.overflowed) a.overflowed = true;
            add_wide(a, b.wide);
            a.non_empty |= b.non_empty;
        }
    }
    return VR_OK;
}

void orc_agg_destroy(orc_agg* a) { delete a; }

int orc_agg_key_dictionary(const orc_agg* a, int32_t key, int32_t* size, int32_t* offsets, uint8_t* data,
                           int64_t data_cap, int64_t* data_bytes) {
    if (!a || !size || key < 0 || key >= (int32_t)a->keys.size()) return VR_ERR_INVALID;
    const auto& strs = a->dict_strings[key];
    *size = (int32_t)strs.size();
    int64_t total = 0;
    for (auto& s : strs) total += (int64_t)s.size();
    if (data_bytes) *data_bytes = total;
    if (data && data_cap < total) return VR_ERR_INVALID;
    int64_t off = 0;
    for (size_t i = 0; i < strs.size(); ++i) {
        if (offsets) offsets[i] = (int32_t)off;
        if (data) std::memcpy(data + off, strs[i].data(), strs[i].size());
        off += (int64_t)strs[i].size();
    }
    if (offsets) offsets[strs.size()] = (int32_t)off;
    return VR_OK;
}
const char* orc_last_error(void) { return g_err.c_str(); }

int orc_hash_rows(int32_t nk, const vr_column_type* types, const vr_column* keys, int64_t n, uint32_t* out,
                  int32_t fin) {
    for (int k = 0; k < nk; ++k) {
        if (types[k].lane == VR_DICT32 && !keys[k].dictionary) return fail(nullptr, VR_ERR_INVALID, "dictionary key without its dictionary");
        if (types[k].lane == VR_UTF8 && !keys[k].offsets) return fail(nullptr, VR_ERR_INVALID, "UTF8 key without offsets");
    }
    for (int64_t i = 0; i < n; ++i) {
        uint32_t h = SEED;
        for (int k = 0; k < nk; ++k) {
            const vr_column& c = keys[k];
            uint32_t v;
            if (c.validity && !bit(c.validity, i)) {
                v = NULL_MARK;
            } else if (types[k].lane == VR_UTF8) {  // mixUtf8 (HashKernels.java:199-213)
                const int32_t o = c.offsets[i];
                v = hash_bytes((const uint8_t*)c.data + o, c.offsets[i + 1] - o);
            } else if (types[k].lane == VR_DICT32) {  // mixDictionary (HashKernels.java:215-236)
                const vr_dictionary& d = *c.dictionary;
                const int32_t id = ((const int32_t*)c.data)[i];
                if (id < 0 || id >= d.size) return fail(nullptr, VR_ERR_INVALID, "dictionary id outside its dictionary");
                v = d.validity && !bit(d.validity, id) ? NULL_MARK
                                                       : hash_bytes(d.data + d.offsets[id], d.offsets[id + 1] - d.offsets[id]);
            } else {
                v = key_hash_value(types[k].lane, key_at(types[k], c, i));
            }
            h = mix32(h, v);
        }
        out[i] = fin ? finish(h) : h;
    }
    return VR_OK;
}

// Rows split into `threads` contiguous partitions (one Spark task each), each
// aggregated in `chunk` batches into its own table; parts[0] ends up holding
// every partition's groups (the reference merges task partials in the Final
// aggregate). Returns the first failing status.
static int run_partitions(const vr_agg_spec* spec, const vr_batch* b, int32_t threads, int64_t chunk,
                          std::vector<orc_agg*>& parts) {
    const int64_t n = b->num_rows;
    parts.assign(threads, nullptr);
    for (int t = 0; t < threads; ++t)
        if (orc_agg_create(spec, &parts[t]) != VR_OK) return VR_ERR_INVALID;
    std::atomic<int> status(VR_OK);
    std::vector<std::thread> ws;
    for (int t = 0; t < threads; ++t) {
        ws.emplace_back([&, t] {
            int64_t lo = n * t / threads, hi = n * (t + 1) / threads;
            // the partition as its own batch: columns offset to `lo`
            std::vector<vr_column> cols(spec->num_columns);
            // bitmaps cannot be offset by arbitrary rows: partitions start on byte boundaries
            int64_t lo8 = lo & ~7ll;
            for (int c = 0; c < spec->num_columns; ++c) {
                const vr_column_type& ty = spec->columns[c];
                int w = ty.lane == VR_INT32 || ty.lane == VR_DICT32 ? 4 : ty.lane == VR_DECIMAL128 ? 16 : 8;
                cols[c].data = (const char*)b->columns[c].data + (ty.lane == VR_BOOL ? lo8 / 8 : lo8 * w);
                cols[c].validity = b->columns[c].validity ? b->columns[c].validity + lo8 / 8 : nullptr;
            }
            vr_batch pb = *b;
            pb.columns = cols.data();
            pb.selection = b->selection ? b->selection + lo8 / 8 : nullptr;
            pb.num_rows = hi - lo8;
            // rows [lo8, lo) belong to the previous partition: select them out
            std::vector<uint8_t> sel;
            if (lo8 < lo || b->selection) {
                sel.assign((size_t)(pb.num_rows + 7) / 8, 0xff);
                for (int64_t r = 0; r < pb.num_rows; ++r) {
                    bool on = (lo8 + r >= lo) && (!b->selection || bit(b->selection, lo8 + r));
                    set_bit(sel.data(), r, on);
                }
                pb.selection = sel.data();
            }
            int rc = orc_agg_update(parts[t], &pb, chunk);
            if (rc != VR_OK) status = rc;
        });
    }
    for (auto& w : ws) w.join();
    for (int t = 1; t < threads; ++t) orc_agg_merge(parts[0], parts[t]);
    return status.load();
}

int orc_agg_run_threads(const vr_agg_spec* spec, const vr_batch* b, int32_t threads, int64_t chunk, double* seconds,
                        int64_t* groups) {
    if (!spec || !b || threads < 1) return VR_ERR_INVALID;
    std::vector<orc_agg*> parts;
    auto t0 = std::chrono::steady_clock::now();
    int rc = run_partitions(spec, b, threads, chunk, parts);
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (groups) *groups = parts[0] ? parts[0]->size : 0;
    for (auto* p : parts) orc_agg_destroy(p);
    return rc;
}

int orc_agg_update_threads(orc_agg* dst, const vr_batch* b, int32_t threads, int64_t chunk) {
    if (!dst || !b || threads < 1) return VR_ERR_INVALID;
    std::vector<orc_agg*> parts;
    int rc = run_partitions(&dst->spec, b, threads, chunk, parts);
    if (rc == VR_OK && parts[0]) rc = orc_agg_merge(dst, parts[0]);
    for (auto* p : parts) orc_agg_destroy(p);
    return rc;
}

}  // extern "C"
