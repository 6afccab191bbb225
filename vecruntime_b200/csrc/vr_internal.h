// Internal descriptors shared by the host side of libvrgpu (abi.cu) and the
// device kernels (agg_kernels.cu). Nothing here crosses the C ABI.
//
// An aggregate spec (vr_agg_spec) compiles into a Program:
//   * a key packing: every key column gets a bit range inside KW 64-bit key
//     words, plus a null bit when nullable; an occupancy bit marks used slots
//     (zeroed memory == empty table);
//   * a list of accumulator Ops, each owning a few 64-bit accumulator words
//     whose identity value is 0, so a table is initialised by a memset;
//   * per accumulator word a combine kind (add / max / or / compensated f64),
//     used both to apply one row's contribution and to merge a whole state
//     (shared-memory tier flush, rehash, partial merges).
#pragma once
#ifndef __CUDACC_RTC__
#include <stdint.h>
#endif

#include "vrgpu.h"

namespace vr {

constexpr int kMaxCols = 16;        // staged input columns per program
constexpr int kMaxKeys = 8;
constexpr int kMaxOps = 24;
constexpr int kMaxAccWords = 120;
constexpr int kMaxKW = 4;           // packed key words
constexpr int kMaxContrib = 8;      // accumulator words one op touches
constexpr int kMaxOut = 48;         // output columns

// How an accumulator word is combined with a contribution.
enum WordKind : uint8_t {
    WK_ADD = 0,      // 64-bit integer add (counts, carry-save limbs)
    WK_MAX = 1,      // unsigned 64-bit max of an order-preserving key
    WK_OR = 2,       // flag bits
    WK_F64 = 3,      // double sum; the next word holds its compensation
    WK_F64C = 4,     // compensation word of a WK_F64 pair
    WK_MAX128 = 5,   // low word of an order-preserving 128-bit key; the next word is the high one
    WK_MAX128L = 6,  // high word of a WK_MAX128 pair
};

enum OpKind : uint8_t {
    OP_COUNT_ROWS = 0,  // 1 word: selected rows
    OP_COUNT_VALID,     // 1 word: rows whose input is valid
    OP_SUM_I32,         // 1 word: sum of an INT32 lane (exact below 2^32 rows)
    OP_SUM_I64,         // 2 words carry-save: sum of low 32 bits, sum of high 32 bits (signed)
    OP_SUM_F64,         // 2 words: compensated double sum
    OP_SUM_D128,        // 4 words carry-save 32-bit limbs (limb 3 signed) of a DECIMAL128 lane
    OP_SUM_PROD,        // 8 words: exact product of terms; 2 carry-save words while it fits
                        //   int64, 4 limb words when it does not (the speculative product),
                        //   an ANSI error flag and the count of non-null products
    OP_MAX_KEY,         // 1 word: max of an order-preserving 64-bit key (min stored complemented)
    OP_MAX_D128,        // 2 words: order-preserving 128-bit key (min stored complemented)
    OP_MERGE_DSUM,      // 5 words: (sum DECIMAL128, isEmpty BOOL) buffer rows: 4 limbs + flags
    OP_MERGE_DAVG,      // 7 words: (sum DECIMAL128, count INT64) buffer rows: 4 limbs + 2 count + flags
};

enum OpFlags : uint8_t { OPF_MIN = 1 };

// flags word bits of the merge ops
constexpr uint64_t kFlagNonEmpty = 1;
constexpr uint64_t kFlagOverflow = 2;

struct OpDesc {
    uint8_t kind;
    uint8_t lane;     // lane of col
    uint8_t flags;
    uint8_t nwords;
    int8_t col;       // staged column or -1
    int8_t col2;
    int8_t nterms;
    int8_t prec;      // OP_SUM_PROD: product precision (rows reaching 10^prec are null / an error)
    int16_t word;     // first accumulator word
    int16_t hword;    // direct tier: first thread-private hot word
    int8_t term_col[3];
    int8_t term_sign[3];
    int16_t prefix_op;  // three-factor OP_SUM_PROD: 1 + index of an earlier two-factor
                        // OP_SUM_PROD with the same first two factors; 0: none
    int64_t term_add[3];
};

struct KeyField {
    int8_t col;        // staged column
    uint8_t lane;
    int8_t word;       // data placement
    int8_t shift;
    uint8_t bits;      // 1, 32, 64 or 128 (unsigned: 128 does not fit an int8_t)
    int8_t null_word;  // -1 when not nullable
    int8_t null_shift;
    uint8_t remap;     // 1: batches bring dictionaries; ids pass through TileView::remap
    int32_t card;      // direct tier: values of this field including null
    int32_t pad2;
    int64_t mul;       // direct tier: combination multiplier
};

struct Program {
    int32_t num_cols;
    uint8_t col_lane[kMaxCols];
    uint8_t col_width[kMaxCols];    // bytes per row; 0 for bit-packed BOOL
    uint8_t col_nullable[kMaxCols];
    int32_t num_keys;
    KeyField keys[kMaxKeys];
    int32_t kw;                      // key words
    int32_t occ_word;
    int32_t occ_shift;
    int32_t lock_mode;               // kw > 2: claim/publish protocol instead of one CAS
    int32_t aw;                      // accumulator words
    int32_t sw;                      // slot stride in words (kw + aw, even)
    int32_t hw;                      // direct tier: thread-private hot words per group
    int32_t num_ops;
    OpDesc ops[kMaxOps];
    uint8_t word_kind[kMaxAccWords];
    int64_t direct_slots;            // combinations for the direct tier (0: not possible)
};

// Per-launch (per instance, in batched mode) description of one batch.
struct BatchDesc {
    const char* col_data[kMaxCols];
    const uint32_t* col_valid[kMaxCols];  // nullptr: all valid
    const uint32_t* selection;
    int64_t num_rows;
    int64_t tile_begin;      // first tile of this instance in the launch's tile space
    int64_t num_tiles;
    uint64_t* table;         // slots * sw words
    int64_t cap_mask;        // slots - 1 (hash tiers); direct tier: slots
    uint64_t* ctrl;          // control block (see Ctrl*)
    int64_t* deferred;       // row ids that found no slot
    int64_t deferred_cap;
    uint64_t* spill;         // shared-tier slots the HBM table could not take (sw words each)
    int64_t spill_cap;
    const Program* prog;
    int32_t tier;            // kTierDirect / kTierHash
    int32_t smem_slots;      // hash tier: shared-memory cache slots (0 = HBM only)
    int32_t warp_agg;
    int32_t tma;             // bulk copies allowed for this batch
    int32_t s_probes;        // hash tier: shared-memory probe limit (a table holding every
                             // group probes until it finds the key; a hot-key cache gives up soon)
    int32_t pad_;
    const int32_t* col_remap[kMaxCols];  // batch dictionary id -> table id (-1: a null entry)
    int32_t col_remap_n[kMaxCols];       // entries of each map (ids at or past it are bad keys)
};

// control block words
enum Ctrl : int {
    CTRL_NEXT_TILE = 0,   // dynamic tile counter (single-instance launches)
    CTRL_GROUPS = 1,      // groups inserted into the HBM table
    CTRL_DEFERRED = 2,    // rows appended to the deferred list
    CTRL_ERROR = 3,       // error bits (kErr*)
    CTRL_TIMEOUT_WHERE = 4,
    CTRL_EMIT_ERROR = 5,  // emission status (VR_ERR_*)
    CTRL_SPILLED = 6,     // slots appended to the spill list
    CTRL_WORDS = 8,
    // an emission's control block: the value behind its first error
    CTRL_EMIT_VALUE_LO = 2,
    CTRL_EMIT_VALUE_HI = 3,
    CTRL_EMIT_VALUE_TYPE = 4,  // bit 63: recorded; precision << 32 | scale
};
constexpr uint64_t kErrTimeout = 1;
constexpr uint64_t kErrDeferredFull = 2;
constexpr uint64_t kErrLockTimeout = 4;
constexpr uint64_t kErrSpillFull = 8;
constexpr uint64_t kErrBadKey = 16;     // dictionary id outside its declared range
constexpr uint64_t kErrProduct = 32;    // ANSI: a decimal product reached its precision

enum OpFlagsExtra : uint8_t {
    OPF_CHECKED = 2,  // OP_SUM_PROD: product overflow is an error
    OPF_NULLABLE = 4  // some input column of the op is declared nullable (else no validity test)
};

constexpr int kTierDirect = 0;
constexpr int kTierHash = 1;

// Output column kinds for emission.
enum OutKind : uint8_t {
    OUT_KEY = 0,        // key column k
    OUT_COUNT,          // int64 from a count word, never null
    OUT_SUM_LONG,       // int64 from carry-save words (w0,w0+1) or an I32 word; null if count(w1)==0
    OUT_SUM_LONG_NN,    // same, never null (merge counts)
    OUT_SUM_DOUBLE,     // f64 pair at w0; null if count(w1)==0
    OUT_SUM_DOUBLE_NN,  // f64 pair, never null (avg buffers)
    OUT_MINMAX,         // key word w0, presence count w1; lane = input lane
    OUT_MINMAX_D128,    // pair at w0, presence w1
    OUT_DEC_SUM,        // decimal buffer from a sum op at w0 (op kind in aux), count w1
    OUT_IS_EMPTY,       // bool: count(w1)==0, or !nonEmpty flag (merge)
    OUT_DEC_MERGE,      // merged decimal sum (OP_MERGE_DSUM / OP_MERGE_DAVG) at w0
    OUT_MERGE_COUNT,    // int64 from carry-save count words of OP_MERGE_DAVG
    OUT_AVG_DOUBLE,     // f64 pair at w0 divided by the count: carry-save words at w1
                        //   (src_op OP_SUM_I64) or a count word (else); null for a zero count
    OUT_DEC_AVG,        // decimal average: the sum as OUT_DEC_MERGE (src_op OP_MERGE_DAVG) or
                        //   OUT_DEC_SUM (else, count word w1) reads it, over its count, at
                        //   (precision, scale) from the sum's (src_precision, src_scale)
};

enum OutFlags : uint8_t {
    OUTF_CHECKED = 1,          // ANSI long sum
    OUTF_NULL_ON_OVERFLOW = 2,
    OUTF_FINAL = 4,
    OUTF_MIN = 8,
    OUTF_FROM_FLAGS = 16,      // OUT_IS_EMPTY from a merge flags word
    OUTF_ZERO_WHEN_EMPTY = 32, // decimal buffer: zero (valid) for an empty group
    OUTF_NULLCOUNT = 64,       // the count is rows (word 0) minus a null count word
    OUTF_UNGROUPED = 128,      // OUT_DEC_AVG of a merge without grouping keys: the sum is not
                               //   checked against the buffer precision (Spark's ungrouped Final
                               //   keeps it in a local that nothing re-checks, VectorAggregates.scala:594-603)
};

struct OutDesc {
    uint8_t kind;
    uint8_t lane;      // output lane
    uint8_t flags;
    uint8_t src_op;    // op kind feeding it (OUT_DEC_SUM, OUT_SUM_LONG)
    int16_t w0;
    int16_t w1;
    int16_t w2;
    int8_t key;        // OUT_KEY: key field
    int8_t pad;
    int32_t precision;
    int32_t scale;
    int16_t src_precision;  // OUT_DEC_AVG: the sum buffer's type
    int16_t src_scale;
};

struct EmitProgram {
    int32_t num_out;
    OutDesc outs[kMaxOut];
};

}  // namespace vr
