// Spec compiler (see plan.h). Maps the reference's aggregate functions onto
// accumulator ops and Spark buffer outputs:
//   CountAgg            VectorAggregates.scala:906-926    COUNT_ROWS / COUNT_VALID -> bigint
//   SumLongAgg          VectorAggregates.scala:142-200    SUM_I32 / SUM_I64 + count -> bigint, null if empty
//   SumDoubleAgg        VectorAggregates.scala:118-136    SUM_F64 + count -> double, null if empty
//   AverageAgg          VectorAggregates.scala:1021-1039  SUM_F64 + count -> (double, bigint)
//   MinMaxAgg           VectorAggregates.scala:929-1018   MAX_KEY / MAX_D128 + count -> value, null if none
//   WideDecimalSumAgg   VectorAggregates.scala:318-395    SUM_I64 / SUM_D128 / SUM_PROD + count -> (decimal, isEmpty)
//   WideDecimalAvgAgg   VectorAggregates.scala:444-516    same sums + count -> (decimal, bigint)
//   CountMergeAgg       VectorAggregates.scala:1042-1059  SUM_I64 of the counts -> bigint
//   AverageMergeAgg     VectorAggregates.scala:1065-1090  SUM_F64 + SUM_I64 -> (double, bigint)
//   WideDecimalSumMergeAgg VectorAggregates.scala:658-781 MERGE_DSUM -> (decimal, isEmpty)
//   WideDecimalAvgMergeAgg VectorAggregates.scala:526-642 MERGE_DAVG -> (decimal, bigint)
#include "plan.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <tuple>

namespace vr {

namespace {

int lane_width(int lane) {
    switch (lane) {
        case VR_INT32:
        case VR_DICT32: return 4;
        case VR_INT64:
        case VR_FLOAT64: return 8;
        case VR_DECIMAL128: return 16;
        case VR_BOOL: return 0;  // bit-packed
    }
    return -1;
}

int bits_for(int n) {  // bits to hold values 0..n-1
    int b = 1;
    while ((1ll << b) < n) ++b;
    return b;
}

struct Builder {
    const vr_agg_spec& spec;
    Plan& plan;
    std::map<std::tuple<int, int, int, int, int, int, int, int64_t, int64_t, int64_t>, int> op_index;
    int words = 0;
    bool full = false;  // op or accumulator capacity exceeded

    Builder(const vr_agg_spec& s, Plan& p) : spec(s), plan(p) {}

    int fail(int code, const std::string& why) {
        plan.reason = why;
        return code;
    }

    int stage(int spec_col) {
        int& st = plan.staged_of_spec[spec_col];
        if (st < 0) {
            Program& P = plan.prog;
            st = P.num_cols++;
            const vr_column_type& t = spec.columns[spec_col];
            P.col_lane[st] = (uint8_t)t.lane;
            P.col_width[st] = (uint8_t)lane_width(t.lane);
            P.col_nullable[st] = (uint8_t)(t.nullable ? 1 : 0);
            plan.spec_of_staged.push_back(spec_col);
        }
        return st;
    }

    static int op_words(int kind) {
        switch (kind) {
            case OP_COUNT_ROWS:
            case OP_COUNT_VALID:
            case OP_SUM_I32:
            case OP_MAX_KEY: return 1;
            case OP_SUM_I64:
            case OP_SUM_F64:
            case OP_MAX_D128: return 2;
            case OP_SUM_D128: return 4;
            case OP_MERGE_DSUM: return 5;
            case OP_MERGE_DAVG: return 7;
            case OP_SUM_PROD: return 8;
        }
        return 0;
    }

    // Adds (or reuses) an op; returns its first accumulator word.
    int add_op(int kind, int col, int col2, int flags, const vr_agg_fn* terms_fn) {
        Program& P = plan.prog;
        int nterms = terms_fn ? terms_fn->num_terms : 0;
        int tc[3] = {-1, -1, -1};
        int ts[3] = {0, 0, 0};
        int64_t ta[3] = {0, 0, 0};
        for (int t = 0; t < nterms; ++t) {
            tc[t] = stage(terms_fn->terms[t].column);
            ts[t] = terms_fn->terms[t].sign < 0 ? -1 : 1;
            ta[t] = terms_fn->terms[t].addend;
        }
        int scol = col >= 0 ? stage(col) : -1;
        int scol2 = col2 >= 0 ? stage(col2) : -1;
        // A count of a non-nullable input is a count of rows.
        if (kind == OP_COUNT_VALID) {
            bool nullable = false;
            if (nterms > 0) {
                for (int t = 0; t < nterms; ++t) nullable |= P.col_nullable[tc[t]] != 0;
            } else {
                nullable = P.col_nullable[scol] != 0;
            }
            if (!nullable) return 0;  // COUNT_ROWS is always op 0, word 0
        }
        {
            bool nullable = false;
            for (int t = 0; t < nterms; ++t) nullable |= P.col_nullable[tc[t]] != 0;
            if (scol >= 0) nullable |= P.col_nullable[scol] != 0;
            if (scol2 >= 0) nullable |= P.col_nullable[scol2] != 0;
            if (nullable) flags |= OPF_NULLABLE;
        }
        int keyflags = flags | ((terms_fn ? terms_fn->product_precision : 0) << 8);
        auto key = std::make_tuple(kind, scol, scol2, keyflags, tc[0] * 4096 + tc[1] * 64 + tc[2], ts[0] * 9 + ts[1] * 3 + ts[2],
                                   nterms, ta[0], ta[1], ta[2]);
        auto it = op_index.find(key);
        if (it != op_index.end()) return P.ops[it->second].word;
        if (P.num_ops >= kMaxOps) {
            full = true;
            return 0;
        }
        int nw = op_words(kind);
        // 128-bit CAS targets must be 16-byte aligned inside the slot
        if (kind == OP_MAX_D128 && ((P.kw + words) & 1)) {
            P.word_kind[words++] = WK_ADD;  // padding word, never touched
        }
        if (words + nw > kMaxAccWords) {
            full = true;
            return 0;
        }
        OpDesc& o = P.ops[P.num_ops];
        std::memset(&o, 0, sizeof(o));
        o.kind = (uint8_t)kind;
        o.lane = scol >= 0 ? P.col_lane[scol] : 0;
        o.flags = (uint8_t)flags;
        o.nwords = (uint8_t)nw;
        o.col = (int8_t)scol;
        o.col2 = (int8_t)scol2;
        o.nterms = (int8_t)nterms;
        o.prec = (int8_t)(terms_fn && terms_fn->product_precision > 0 ? std::min(38, terms_fn->product_precision) : 38);
        o.word = (int16_t)words;
        for (int t = 0; t < 3; ++t) {
            o.term_col[t] = (int8_t)tc[t];
            o.term_sign[t] = (int8_t)ts[t];
            o.term_add[t] = ta[t];
        }
        uint8_t* wk = P.word_kind + words;
        switch (kind) {
            case OP_COUNT_ROWS:
            case OP_COUNT_VALID:
            case OP_SUM_I32: wk[0] = WK_ADD; break;
            case OP_SUM_I64: wk[0] = wk[1] = WK_ADD; break;
            case OP_SUM_F64: wk[0] = WK_F64; wk[1] = WK_F64C; break;
            case OP_SUM_D128: for (int i = 0; i < 4; ++i) wk[i] = WK_ADD; break;
            case OP_SUM_PROD: for (int i = 0; i < 6; ++i) wk[i] = WK_ADD; wk[6] = WK_OR; wk[7] = WK_ADD; break;
            case OP_MAX_KEY: wk[0] = WK_MAX; break;
            case OP_MAX_D128: wk[0] = WK_MAX128; wk[1] = WK_MAX128L; break;
            case OP_MERGE_DSUM: for (int i = 0; i < 4; ++i) wk[i] = WK_ADD; wk[4] = WK_OR; break;
            case OP_MERGE_DAVG: for (int i = 0; i < 6; ++i) wk[i] = WK_ADD; wk[6] = WK_OR; break;
        }
        op_index[key] = P.num_ops;
        ++P.num_ops;
        words += nw;
        return o.word;
    }

    OutDesc* last_out = nullptr;

    // A decimal average's result type: given, or Spark's Decimal(p + 4, s + 4)
    // of the input decimal(p, s) behind the Decimal(p + 10, s) buffer, bounded
    // to 38 (Average.resultType; DecimalType.bounded).
    int avg_result_type(const vr_agg_fn& f, int& rp, int& rs) {
        if (f.result_precision > 0) {
            rp = f.result_precision;
            rs = f.result_scale;
        } else {
            if (f.precision >= 38) return fail(VR_ERR_INVALID, "a 38-digit average buffer needs its result type");
            rp = std::min(f.precision - 10 + 4, 38);
            rs = std::min(f.scale + 4, 38);
        }
        if (rp < 1 || rp > 38 || rs < f.scale || rs > rp) return fail(VR_ERR_UNSUPPORTED, "decimal average result type");
        return VR_OK;
    }

    void out(uint8_t kind, int lane, int flags, int src_op, int w0, int w1, int key, int precision, int scale) {
        EmitProgram& E = plan.emit;
        OutDesc& d = E.outs[E.num_out++];
        std::memset(&d, 0, sizeof(d));
        d.kind = kind;
        d.lane = (uint8_t)lane;
        d.flags = (uint8_t)flags;
        d.src_op = (uint8_t)src_op;
        d.w0 = (int16_t)w0;
        d.w1 = (int16_t)w1;
        d.key = (int8_t)key;
        d.precision = precision;
        d.scale = scale;
        last_out = &d;
        vr_column_type t;
        std::memset(&t, 0, sizeof(t));
        t.lane = lane;
        t.precision = (lane == VR_DECIMAL128 || precision > 0) ? precision : 0;
        t.scale = scale;
        t.nullable = 1;
        plan.out_types.push_back(t);
    }

    int layout_keys() {
        Program& P = plan.prog;
        P.num_keys = spec.num_keys;
        struct Field {
            int idx, lane, bits, nullable;
        };
        std::vector<Field> fs;
        for (int k = 0; k < spec.num_keys; ++k) {
            int c = spec.key_columns[k];
            if (c < 0 || c >= spec.num_columns) return fail(VR_ERR_INVALID, "key column out of range");
            const vr_column_type& t = spec.columns[c];
            int bits;
            switch (t.lane) {
                case VR_INT32: bits = 32; break;
                case VR_DICT32: bits = t.dict_size > 0 ? std::min(32, bits_for(t.dict_size)) : 32; break;
                case VR_INT64:
                case VR_FLOAT64: bits = 64; break;
                case VR_BOOL: bits = 1; break;
                case VR_DECIMAL128: bits = 128; break;
                default: return fail(VR_ERR_UNSUPPORTED, "key lane not supported on the GPU");
            }
            fs.push_back({k, t.lane, bits, t.nullable ? 1 : 0});
        }
        // Direct tier: every key a dictionary id or boolean with a known domain.
        bool direct = true;
        int64_t combos = 1;
        for (auto& f : fs) {
            const vr_column_type& t = spec.columns[spec.key_columns[f.idx]];
            int card;
            if (f.lane == VR_BOOL)
                card = 2;
            else if (f.lane == VR_DICT32 && t.dict_size > 0)
                card = t.dict_size;
            else {
                direct = false;
                break;
            }
            card += f.nullable;
            combos *= card;
            if (combos > (1 << 20)) {
                direct = false;
                break;
            }
        }
        plan.direct_ok = direct;
        P.direct_slots = direct ? combos : 0;

        // Single non-nullable 64-bit key: sentinel layout, one word.
        if (fs.size() == 1 && fs[0].bits == 64 && !fs[0].nullable) {
            P.kw = 1;
            P.occ_word = -1;
            P.occ_shift = 0;
            KeyField& kf = P.keys[0];
            std::memset(&kf, 0, sizeof(kf));
            kf.col = (int8_t)stage(spec.key_columns[0]);
            kf.lane = (uint8_t)fs[0].lane;
            kf.word = 0;
            kf.shift = 0;
            kf.bits = 64;
            kf.null_word = -1;
        } else {
            // dedicated words for 128/64-bit data; small words (62 usable bits) for the rest
            int dedicated = 0;
            for (auto& f : fs) dedicated += f.bits == 128 ? 2 : (f.bits == 64 ? 1 : 0);
            std::vector<int> small_used;  // next free bit per small word
            auto place_small = [&](int bits) {
                for (size_t i = 0; i < small_used.size(); ++i) {
                    if (small_used[i] + bits <= 62) {
                        int sh = small_used[i];
                        small_used[i] += bits;
                        return std::make_pair((int)i, sh);
                    }
                }
                small_used.push_back(bits);
                return std::make_pair((int)small_used.size() - 1, 0);
            };
            int next_ded = 0;
            for (auto& f : fs) {
                KeyField& kf = P.keys[f.idx];
                std::memset(&kf, 0, sizeof(kf));
                kf.col = (int8_t)stage(spec.key_columns[f.idx]);
                kf.lane = (uint8_t)f.lane;
                kf.bits = (uint8_t)f.bits;
                kf.null_word = -1;
                if (f.bits >= 64) {
                    kf.word = (int8_t)next_ded;
                    kf.shift = 0;
                    next_ded += f.bits / 64;
                }
            }
            for (auto& f : fs) {  // small data fields
                if (f.bits >= 64) continue;
                auto ws = place_small(f.bits);
                KeyField& kf = P.keys[f.idx];
                kf.word = (int8_t)(dedicated + ws.first);
                kf.shift = (int8_t)ws.second;
            }
            for (auto& f : fs) {  // null bits
                if (!f.nullable) continue;
                auto ws = place_small(1);
                KeyField& kf = P.keys[f.idx];
                kf.null_word = (int8_t)(dedicated + ws.first);
                kf.null_shift = (int8_t)ws.second;
            }
            if (small_used.empty()) small_used.push_back(0);  // a word for the occupancy bit
            P.kw = dedicated + (int)small_used.size();
            P.occ_word = P.kw - 1;  // small words follow dedicated ones: bits 62-63 free
            P.occ_shift = 63;
        }
        if (P.kw > kMaxKW) return fail(VR_ERR_UNSUPPORTED, "grouping key wider than 256 bits");
        // keys whose batches bring their own dictionaries go through a map to table ids
        for (auto& f : fs) {
            const vr_column_type& t = spec.columns[spec.key_columns[f.idx]];
            if (!(t.flags & VR_COL_BATCH_DICTIONARY)) continue;
            if (t.lane != VR_DICT32) return fail(VR_ERR_INVALID, "only VR_DICT32 keys bring batch dictionaries");
            P.keys[f.idx].remap = 1;
        }
        P.lock_mode = P.kw > 1 ? 1 : 0;
        // direct tier: combination multipliers
        if (direct) {
            int64_t mul = 1;
            for (auto& f : fs) {
                const vr_column_type& t = spec.columns[spec.key_columns[f.idx]];
                KeyField& kf = P.keys[f.idx];
                int card = (f.lane == VR_BOOL ? 2 : t.dict_size) + f.nullable;
                kf.card = card;
                kf.mul = mul;
                mul *= card;
            }
        }
        return VR_OK;
    }

    int build() {
        Program& P = plan.prog;
        std::memset(&P, 0, sizeof(P));
        std::memset(&plan.emit, 0, sizeof(plan.emit));
        plan.staged_of_spec.assign(spec.num_columns, -1);
        plan.spec_of_staged.clear();
        plan.out_types.clear();
        if (spec.num_columns < 0 || spec.num_columns > 64) return fail(VR_ERR_INVALID, "bad column count");
        if (spec.num_keys < 0 || spec.num_keys > kMaxKeys) return fail(VR_ERR_UNSUPPORTED, "too many grouping keys");
        if (spec.num_fns < 0 || spec.num_fns > 32) return fail(VR_ERR_UNSUPPORTED, "too many functions");
        for (int c = 0; c < spec.num_columns; ++c)
            if (lane_width(spec.columns[c].lane) < 0) return fail(VR_ERR_UNSUPPORTED, "unknown lane type");
        int rc = layout_keys();
        if (rc != VR_OK) return rc;
        if (P.num_cols > kMaxCols) return fail(VR_ERR_UNSUPPORTED, "too many input columns");
        // op 0 is always COUNT_ROWS at word 0: occupancy and count(*)
        add_op(OP_COUNT_ROWS, -1, -1, 0, nullptr);

        for (int k = 0; k < spec.num_keys; ++k) {
            const vr_column_type& t = spec.columns[spec.key_columns[k]];
            out(OUT_KEY, t.lane == VR_DICT32 ? VR_DICT32 : t.lane, 0, 0, 0, 0, k, t.precision, t.scale);
        }
        auto col_ok = [&](int c) { return c >= 0 && c < spec.num_columns; };
        for (int i = 0; i < spec.num_fns; ++i) {
            const vr_agg_fn& f = spec.fns[i];
            const vr_column_type* in = col_ok(f.input) ? &spec.columns[f.input] : nullptr;
            const vr_column_type* in2 = col_ok(f.input2) ? &spec.columns[f.input2] : nullptr;
            bool checked = (f.flags & VR_FN_CHECKED) != 0;
            int dflags = ((f.flags & VR_FN_FINAL) ? OUTF_FINAL : OUTF_ZERO_WHEN_EMPTY) |
                         ((f.flags & VR_FN_NULL_ON_OVERFLOW) ? OUTF_NULL_ON_OVERFLOW : 0);
            switch (f.kind) {
                case VR_FN_COUNT_STAR:
                    out(OUT_COUNT, VR_INT64, 0, 0, 0, 0, -1, 0, 0);
                    break;
                case VR_FN_COUNT: {
                    if (!in) return fail(VR_ERR_INVALID, "count needs an input column");
                    int w = add_op(OP_COUNT_VALID, f.input, -1, 0, nullptr);
                    out(OUT_COUNT, VR_INT64, 0, 0, w, 0, -1, 0, 0);
                    break;
                }
                case VR_FN_SUM_LONG: {
                    if (!in || (in->lane != VR_INT32 && in->lane != VR_INT64))
                        return fail(VR_ERR_UNSUPPORTED, "sum(long) needs an INT32 or INT64 input");
                    int kind = in->lane == VR_INT32 ? OP_SUM_I32 : OP_SUM_I64;
                    int w = add_op(kind, f.input, -1, 0, nullptr);
                    int c = add_op(OP_COUNT_VALID, f.input, -1, 0, nullptr);
                    out(OUT_SUM_LONG, VR_INT64, checked ? OUTF_CHECKED : 0, kind, w, c, -1, 0, 0);
                    break;
                }
                case VR_FN_SUM_DOUBLE:
                case VR_FN_AVG_DOUBLE: {
                    if (!in || in->lane != VR_FLOAT64) return fail(VR_ERR_UNSUPPORTED, "double sum needs a FLOAT64 input");
                    int w = add_op(OP_SUM_F64, f.input, -1, 0, nullptr);
                    int c = add_op(OP_COUNT_VALID, f.input, -1, 0, nullptr);
                    if (f.kind == VR_FN_SUM_DOUBLE) {
                        out(OUT_SUM_DOUBLE, VR_FLOAT64, 0, 0, w, c, -1, 0, 0);
                    } else if (f.flags & VR_FN_FINAL) {  // Complete: the average itself, then the count
                        out(OUT_AVG_DOUBLE, VR_FLOAT64, 0, 0, w, c, -1, 0, 0);
                        out(OUT_COUNT, VR_INT64, 0, 0, c, 0, -1, 0, 0);
                    } else {
                        out(OUT_SUM_DOUBLE_NN, VR_FLOAT64, 0, 0, w, c, -1, 0, 0);
                        out(OUT_COUNT, VR_INT64, 0, 0, c, 0, -1, 0, 0);
                    }
                    break;
                }
                case VR_FN_MIN:
                case VR_FN_MAX: {
                    if (!in) return fail(VR_ERR_INVALID, "min/max needs an input column");
                    int mflag = f.kind == VR_FN_MIN ? OPF_MIN : 0;
                    int oflag = f.kind == VR_FN_MIN ? OUTF_MIN : 0;
                    int c = add_op(OP_COUNT_VALID, f.input, -1, 0, nullptr);
                    if (in->lane == VR_DECIMAL128) {
                        int w = add_op(OP_MAX_D128, f.input, -1, mflag, nullptr);
                        c = add_op(OP_COUNT_VALID, f.input, -1, 0, nullptr);
                        out(OUT_MINMAX_D128, VR_DECIMAL128, oflag, 0, w, c, -1, in->precision, in->scale);
                    } else if (in->lane == VR_INT32 || in->lane == VR_INT64 || in->lane == VR_FLOAT64) {
                        int w = add_op(OP_MAX_KEY, f.input, -1, mflag, nullptr);
                        out(OUT_MINMAX, in->lane, oflag, 0, w, c, -1, in->precision, in->scale);
                    } else {
                        return fail(VR_ERR_UNSUPPORTED, "min/max lane not supported on the GPU");
                    }
                    break;
                }
                case VR_FN_SUM_DECIMAL:
                case VR_FN_AVG_DECIMAL: {
                    if (f.precision < 1 || f.precision > 38) return fail(VR_ERR_INVALID, "decimal buffer precision");
                    int rp = 0, rs = 0;
                    if (f.kind == VR_FN_AVG_DECIMAL && (f.flags & VR_FN_FINAL)) {
                        int rc2 = avg_result_type(f, rp, rs);
                        if (rc2 != VR_OK) return rc2;
                    }
                    int kind, w, c;
                    if (f.num_terms > 0) {
                        if (f.num_terms < 2 || f.num_terms > 3) return fail(VR_ERR_INVALID, "product needs 2 or 3 terms");
                        int scale = 0;
                        for (int t = 0; t < f.num_terms; ++t) {
                            int tc = f.terms[t].column;
                            if (!col_ok(tc) || spec.columns[tc].lane != VR_INT64)
                                return fail(VR_ERR_UNSUPPORTED, "product terms must be INT64 decimal lanes");
                            scale += spec.columns[tc].scale;
                        }
                        if (scale != f.scale)
                            return fail(VR_ERR_UNSUPPORTED, "product needs rounding (scale adjustment) - CPU path");
                        kind = OP_SUM_PROD;
                        w = add_op(kind, -1, -1, (f.flags & VR_FN_CHECKED) ? OPF_CHECKED : 0, &f);
                        c = w + 7;  // the op counts its null products: count = rows - nulls
                    } else {
                        if (!in) return fail(VR_ERR_INVALID, "decimal sum needs an input");
                        if (in->lane == VR_INT64 || in->lane == VR_INT32)
                            kind = OP_SUM_I64;
                        else if (in->lane == VR_DECIMAL128)
                            kind = OP_SUM_D128;
                        else
                            return fail(VR_ERR_UNSUPPORTED, "decimal sum lane");
                        w = add_op(kind, f.input, -1, 0, nullptr);
                        c = add_op(OP_COUNT_VALID, f.input, -1, 0, nullptr);
                    }
                    const int nc = kind == OP_SUM_PROD ? OUTF_NULLCOUNT : 0;  // products count their nulls
                    if (f.kind == VR_FN_SUM_DECIMAL) {
                        out(OUT_DEC_SUM, VR_DECIMAL128, dflags | nc, kind, w, c, -1, f.precision, f.scale);
                        out(OUT_IS_EMPTY, VR_BOOL, nc, 0, 0, c, -1, 0, 0);
                    } else if (f.flags & VR_FN_FINAL) {  // Complete: the average at its result type
                        out(OUT_DEC_AVG, rp <= 18 ? VR_INT64 : VR_DECIMAL128,
                            nc | ((f.flags & VR_FN_NULL_ON_OVERFLOW) ? OUTF_NULL_ON_OVERFLOW : 0), kind, w, c, -1, rp, rs);
                        last_out->src_precision = (int16_t)f.precision;
                        last_out->src_scale = (int16_t)f.scale;
                        out(OUT_COUNT, VR_INT64, nc, 0, c, 0, -1, 0, 0);
                    } else {
                        out(OUT_DEC_SUM, VR_DECIMAL128, OUTF_ZERO_WHEN_EMPTY | nc, kind, w, c, -1, f.precision,
                            f.scale);
                        out(OUT_COUNT, VR_INT64, nc, 0, c, 0, -1, 0, 0);
                    }
                    break;
                }
                case VR_FN_COUNT_MERGE: {
                    if (!in || in->lane != VR_INT64) return fail(VR_ERR_UNSUPPORTED, "count merge needs an INT64 buffer");
                    int w = add_op(OP_SUM_I64, f.input, -1, 0, nullptr);
                    out(OUT_SUM_LONG_NN, VR_INT64, 0, OP_SUM_I64, w, 0, -1, 0, 0);
                    break;
                }
                case VR_FN_AVG_DOUBLE_MERGE: {
                    if (!in || !in2 || in->lane != VR_FLOAT64 || in2->lane != VR_INT64)
                        return fail(VR_ERR_UNSUPPORTED, "avg merge needs (FLOAT64, INT64) buffers");
                    int ws = add_op(OP_SUM_F64, f.input, -1, 0, nullptr);
                    int wc = add_op(OP_SUM_I64, f.input2, -1, 0, nullptr);
                    if (f.flags & VR_FN_FINAL)  // Final: sum / count, null when no row counted
                        out(OUT_AVG_DOUBLE, VR_FLOAT64, 0, OP_SUM_I64, ws, wc, -1, 0, 0);
                    else
                        out(OUT_SUM_DOUBLE_NN, VR_FLOAT64, 0, 0, ws, 0, -1, 0, 0);
                    out(OUT_SUM_LONG_NN, VR_INT64, 0, OP_SUM_I64, wc, 0, -1, 0, 0);
                    break;
                }
                case VR_FN_SUM_DECIMAL_MERGE: {
                    if (!in || !in2 || in->lane != VR_DECIMAL128 || in2->lane != VR_BOOL)
                        return fail(VR_ERR_UNSUPPORTED, "decimal sum merge needs (DECIMAL128, BOOL) buffers");
                    if (f.precision < 1 || f.precision > 38) return fail(VR_ERR_INVALID, "decimal buffer precision");
                    int w = add_op(OP_MERGE_DSUM, f.input, f.input2, 0, nullptr);
                    int mflags = ((f.flags & VR_FN_FINAL) ? OUTF_FINAL : 0) |
                                 ((f.flags & VR_FN_NULL_ON_OVERFLOW) ? OUTF_NULL_ON_OVERFLOW : 0);
                    out(OUT_DEC_MERGE, VR_DECIMAL128, mflags, OP_MERGE_DSUM, w, 0, -1, f.precision, f.scale);
                    out(OUT_IS_EMPTY, VR_BOOL, OUTF_FROM_FLAGS, 0, 0, w + 4, -1, 0, 0);
                    break;
                }
                case VR_FN_AVG_DECIMAL_MERGE: {
                    if (!in || !in2 || in->lane != VR_DECIMAL128 || in2->lane != VR_INT64)
                        return fail(VR_ERR_UNSUPPORTED, "decimal avg merge needs (DECIMAL128, INT64) buffers");
                    if (f.precision < 1 || f.precision > 38) return fail(VR_ERR_INVALID, "decimal buffer precision");
                    int w = add_op(OP_MERGE_DAVG, f.input, f.input2, 0, nullptr);
                    if (f.flags & VR_FN_FINAL) {  // Final: DecimalAvgResult in the sum slot
                        int rp = 0, rs = 0;
                        int rc2 = avg_result_type(f, rp, rs);
                        if (rc2 != VR_OK) return rc2;
                        out(OUT_DEC_AVG, rp <= 18 ? VR_INT64 : VR_DECIMAL128,
                            ((f.flags & VR_FN_NULL_ON_OVERFLOW) ? OUTF_NULL_ON_OVERFLOW : 0) |
                                (spec.num_keys == 0 ? OUTF_UNGROUPED : 0),
                            OP_MERGE_DAVG, w, w + 4, -1, rp, rs);
                        last_out->src_precision = (int16_t)f.precision;
                        last_out->src_scale = (int16_t)f.scale;
                    } else {
                        out(OUT_DEC_MERGE, VR_DECIMAL128, 0, OP_MERGE_DAVG, w, 0, -1, f.precision, f.scale);
                    }
                    out(OUT_MERGE_COUNT, VR_INT64, 0, 0, w + 4, 0, -1, 0, 0);
                    break;
                }
                default:
                    return fail(VR_ERR_UNSUPPORTED, "aggregate function not supported on the GPU");
            }
            if (full) return fail(VR_ERR_UNSUPPORTED, "too many accumulators");
            if (plan.emit.num_out > kMaxOut - 2) return fail(VR_ERR_UNSUPPORTED, "too many output columns");
        }
        if (P.num_cols > kMaxCols) return fail(VR_ERR_UNSUPPORTED, "too many input columns");
        P.aw = words;
        P.sw = (P.kw + P.aw + 1) & ~1;
        // a three-factor product whose first two factors are an earlier
        // two-factor product's: the direct tier reuses that product
        for (int i = 0; i < P.num_ops; ++i) {
            OpDesc& b = P.ops[i];
            if (b.kind != OP_SUM_PROD || b.nterms != 3) continue;
            for (int k = 0; k < i && !b.prefix_op; ++k) {
                const OpDesc& a = P.ops[k];
                if (a.kind != OP_SUM_PROD || a.nterms != 2) continue;
                bool same = true;
                for (int t = 0; t < 2; ++t)
                    same = same && a.term_col[t] == b.term_col[t] && a.term_sign[t] == b.term_sign[t] &&
                           a.term_add[t] == b.term_add[t];
                if (same) b.prefix_op = (int16_t)(k + 1);
            }
        }
        // direct tier: hot words per op (the running values every row touches)
        P.hw = 0;
        for (int i = 0; i < P.num_ops; ++i) {
            OpDesc& o = P.ops[i];
            int hot = 1;
            if (o.kind == OP_SUM_F64 || o.kind == OP_SUM_D128 || o.kind == OP_MAX_D128) hot = 2;
            if (o.kind == OP_MERGE_DSUM || o.kind == OP_MERGE_DAVG) hot = 3;
            o.hword = (int16_t)P.hw;
            P.hw += hot;
        }
        if (P.direct_slots == 0 && spec.num_keys == 0) P.direct_slots = 1;
        if (spec.num_keys == 0) plan.direct_ok = true;
        return VR_OK;
    }
};

}  // namespace

int compile_plan(const vr_agg_spec& spec, Plan& plan) {
    Builder b(spec, plan);
    int rc = b.build();
    return rc;
}

}  // namespace vr
