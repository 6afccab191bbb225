/*
 * vrgpu.h -- C ABI of the B200 grouped-aggregation backend (libvrgpu.so).
 *
 * One hot path: partial and final grouped aggregation over Arrow-layout
 * batches (key hashing, group probe/insert into an open-addressing table,
 * count/sum/min/max/avg that honour validity bitmaps, exact 128-bit decimal
 * sums with Spark's null and overflow rules).
 *
 * The entry points replace the kernel-level contract of the reference's
 * aggregate operator (vecruntime, Java):
 *   GroupKeyTable.assign(keys, n, outIds, selection)
 *       kernels/src/main/java/io/vecruntime/kernels/GroupKeyTable.java:709-764
 *   GroupedAccumulators.*.update(v, assignment)
 *       kernels/src/main/java/io/vecruntime/kernels/GroupedAccumulators.java:195-1462
 *   GroupKeyTable.writeKeys / GroupedAggState.writeBuffer (emission)
 *       kernels/src/main/java/io/vecruntime/kernels/GroupKeyTable.java:2851-2920
 *       spark/src/main/scala/io/vecruntime/spark/agg/VectorAggregates.scala:54-97
 * as driven by VectorGroupedAggregateIterator.consume / buildBatch
 *       spark/src/main/scala/org/apache/spark/sql/vecruntime/VectorHashAggregateExec.scala:584-602, 831-913
 *
 * Conventions
 *   - Every call returns a status code (VR_OK = 0); nothing throws across
 *     the boundary. After an error other than VR_ERR_INVALID /
 *     VR_ERR_UNSUPPORTED the handle is dead: the caller destroys it (the
 *     Java side closes it, as the reference's task-completion listener does).
 *   - One handle per task thread; a handle is not thread-safe. Many handles
 *     run concurrently, each on its own CUDA stream.
 *   - Buffers are Arrow layout: little-endian values, LSB-first validity
 *     bitmaps starting at bit 0 (NULL = every row valid), DECIMAL128 as two
 *     little-endian int64 limbs (lo at 16*i, hi at 16*i+8), BOOL as a packed
 *     bitmap.
 *   - The caller owns input buffers and keeps them alive (and, for async
 *     copies, pinned: vr_host_alloc / vr_host_register) until vr_agg_sync
 *     returns. The caller owns output buffers. The handle owns device state.
 */
#ifndef VRGPU_H
#define VRGPU_H

#ifndef __CUDACC_RTC__ /* per-spec kernels compiled at run time get these types from their prelude */
#include <stddef.h>
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define VRGPU_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
enum vr_status {
    VR_OK = 0,
    VR_ERR_INVALID = 1,           /* bad argument or spec                        */
    VR_ERR_OOM = 2,               /* device or pinned allocation refused         */
    VR_ERR_OVERFLOW = 3,          /* ANSI bigint sum overflow: Spark's
                                     ARITHMETIC_OVERFLOW (VectorAggregates.scala:145-146) */
    VR_ERR_DECIMAL_PRECISION = 4, /* ANSI decimal result past its precision
                                     (VectorAggregates.scala:333-341)            */
    VR_ERR_TIMEOUT = 5,           /* a bounded device wait gave up               */
    VR_ERR_CUDA = 6,              /* CUDA runtime error; text in vr_agg_last_error */
    VR_ERR_UNSUPPORTED = 7,       /* outside the GPU gate: caller falls back to
                                     the Vector API path, then Spark             */
    VR_ERR_STATE = 8,             /* dead handle or call out of order            */
    VR_ERR_ADMISSION = 9,         /* serving: request larger than the HBM cap    */
    VR_ERR_DECIMAL_OVERFLOW = 10  /* ANSI overflow of a merged decimal sum:
                                     Spark's overflowInSumOfDecimal (VectorAggregates.scala:737-741) */
};

/* ---- lane types (reference VecType, kernels/.../VecType.java:23-64) ---- */
enum vr_lane {
    VR_INT32 = 1,
    VR_INT64 = 2,      /* also DECIMAL(p<=18, s) unscaled (TypeMapping.java:87-90) */
    VR_FLOAT64 = 3,    /* keys group by raw bits (GroupKeyTable.java:2350-2353)    */
    VR_BOOL = 4,       /* bit-packed                                               */
    VR_DECIMAL128 = 5, /* DECIMAL(p>18, s): two LE int64 limbs (Decimal128.java:21-61) */
    VR_DICT32 = 6,     /* dictionary-encoded UTF8: int32 ids into a dictionary of
                          strings (vr_column.dictionary); GroupKeyTable keeps
                          strings as ids (GroupKeyTable.java:27-36)                */
    VR_UTF8 = 7        /* plain UTF8: bytes + n + 1 int32 offsets (vr_hash_rows only) */
};

typedef struct vr_column_type {
    int32_t lane;      /* enum vr_lane                                          */
    int32_t precision; /* decimal precision; 0 when not a decimal               */
    int32_t scale;     /* decimal scale                                         */
    int32_t nullable;  /* 0: the column never carries a validity bitmap         */
    int32_t dict_size; /* VR_DICT32 / VR_BOOL keys: ids lie in [0, dict_size);
                          0 = unknown (no direct indexing). With
                          VR_COL_BATCH_DICTIONARY: the most distinct strings
                          the table keeps for the column                        */
    int32_t flags;     /* enum vr_column_flags                                  */
} vr_column_type;

enum vr_column_flags {
    /* VR_DICT32 key whose batches each bring their own dictionary
     * (vr_column.dictionary, e.g. Parquet row-group dictionaries): the
     * handle maps every batch's entries onto a table dictionary it keeps
     * across batches (GroupKeyTable.toIds, GroupKeyTable.java:1308-1430),
     * keys are emitted as table ids, and vr_agg_key_dictionary returns the
     * table dictionary's strings. A null entry makes its rows null. */
    VR_COL_BATCH_DICTIONARY = 1
};

/* ---- aggregate functions (reference VectorAggFunction implementations) -- */
enum vr_fn_kind {
    VR_FN_COUNT_STAR = 1,      /* CountAgg(None)           VectorAggregates.scala:906-926  */
    VR_FN_COUNT = 2,           /* CountAgg(Some(e))                                        */
    VR_FN_SUM_LONG = 3,        /* SumLongAgg (INT32/INT64) VectorAggregates.scala:142-200  */
    VR_FN_SUM_DOUBLE = 4,      /* SumDoubleAgg             VectorAggregates.scala:118-136  */
    VR_FN_AVG_DOUBLE = 5,      /* AverageAgg (sum, count)  VectorAggregates.scala:1021-1039 */
    VR_FN_MIN = 6,             /* MinMaxAgg(isMin = true)  VectorAggregates.scala:929-1018 */
    VR_FN_MAX = 7,             /* MinMaxAgg(isMin = false)                                 */
    VR_FN_SUM_DECIMAL = 8,     /* WideDecimalSumAgg (sum, isEmpty) VectorAggregates.scala:318-395 */
    VR_FN_AVG_DECIMAL = 9,     /* WideDecimalAvgAgg (sum, count)   VectorAggregates.scala:444-516 */
    VR_FN_COUNT_MERGE = 10,    /* CountMergeAgg            VectorAggregates.scala:1042-1059 */
    VR_FN_AVG_DOUBLE_MERGE = 11,  /* AverageMergeAgg       VectorAggregates.scala:1065-1090 */
    VR_FN_SUM_DECIMAL_MERGE = 12, /* WideDecimalSumMergeAgg VectorAggregates.scala:658-781  */
    VR_FN_AVG_DECIMAL_MERGE = 13  /* WideDecimalAvgMergeAgg VectorAggregates.scala:526-642  */
};
/* A merge of SumLong / SumDouble / MinMax buffers is VR_FN_SUM_LONG /
 * VR_FN_SUM_DOUBLE / VR_FN_MIN / VR_FN_MAX over the buffer column, exactly as
 * compileMerge builds them (VectorAggregates.scala:1197-1215). */

enum vr_fn_flags {
    VR_FN_CHECKED = 1,          /* ANSI bigint sum: overflow -> VR_ERR_OVERFLOW      */
    VR_FN_NULL_ON_OVERFLOW = 2, /* non-ANSI decimal: past precision -> null          */
    VR_FN_FINAL = 4,            /* Final / Complete: the function's result in its first
                                   slot (Spark's evaluateExpression over the merged
                                   buffer): a decimal sum checked against its precision;
                                   avg(double) = sum / count, null for no rows
                                   (Average, VectorAggregates.scala:1065-1090); a decimal
                                   avg = sum / count at the result type with Spark's
                                   half-up division (DecimalAvgResult,
                                   VectorAggregates.scala:405-430). The count stays in
                                   the second slot, as the reference emits it.        */
    VR_FN_STRICT = 8            /* accepted for parity with spark.vecruntime.exec.strictFloatingPoint;
                                   FP64 sums are compensated, not sequential          */
};

/* One factor of a fused decimal product: value = addend + sign * column,
 * unscaled at the column's scale (e.g. (1 - disc) with disc DECIMAL(12,2):
 * addend 100, sign -1). Replaces the reference's SpeculativeDecimalMulExpr
 * (spark/.../expr/DecimalExprs.scala:470-516) in front of a decimal sum. */
typedef struct vr_term {
    int32_t column;
    int32_t sign; /* +1 or -1 */
    int64_t addend;
} vr_term;

typedef struct vr_agg_fn {
    int32_t kind;      /* enum vr_fn_kind                                         */
    int32_t input;     /* input column (-1 for COUNT_STAR); merges: 1st buffer col */
    int32_t input2;    /* merges: 2nd buffer column (count / isEmpty); else -1     */
    int32_t flags;     /* enum vr_fn_flags                                         */
    int32_t precision; /* decimal sum/avg buffer type (Spark: Decimal(p + 10, s))  */
    int32_t scale;
    int32_t num_terms; /* 0: input column; 2..3: exact product of terms[]          */
    int32_t product_precision; /* declared precision of the product (0 = 38): a row
                                  whose exact product reaches 10^p is null (non-ANSI)
                                  or VR_ERR_DECIMAL_PRECISION with VR_FN_CHECKED,
                                  Spark's CheckOverflow on the multiply            */
    vr_term terms[3];
    int32_t result_precision; /* VR_FN_FINAL decimal avg: the result type, Spark's
                                 Decimal(p + 4, s + 4) of the input decimal(p, s),
                                 bounded to 38; 0 = derived from the buffer type
                                 (Decimal(p + 10, s), which must then be below 38) */
    int32_t result_scale;
} vr_agg_fn;

enum vr_spec_flags {
    VR_SPEC_FORCE_GLOBAL = 1,  /* tests / tuning: skip the shared-memory tiers   */
    VR_SPEC_FORCE_SHARED = 2,  /* shared-memory hash table in front of HBM       */
    VR_SPEC_FORCE_DIRECT = 4,  /* direct-indexed thread-private tier             */
    VR_SPEC_NO_WARP_AGG = 8,   /* no __match_any_sync pre-aggregation            */
    VR_SPEC_WARP_AGG = 16,     /* force __match_any_sync pre-aggregation         */
    VR_SPEC_NO_TMA = 32,       /* plain loads instead of bulk copies into smem   */
    VR_SPEC_TRACE = 64,        /* record cudaEvent pairs per H2D / kernel / D2H  */
    VR_SPEC_NO_JIT = 128       /* run the interpreted kernel, not one compiled
                                  for this spec (also: environment VRGPU_JIT=0)  */
};

typedef struct vr_agg_spec {
    int32_t num_columns;            /* input columns per batch                 */
    const vr_column_type* columns;
    int32_t num_keys;               /* 0 = ungrouped (one group)               */
    const int32_t* key_columns;
    int32_t num_fns;
    const vr_agg_fn* fns;
    int64_t est_groups;             /* cardinality estimate; 0 = unknown       */
    int64_t max_batch_rows;         /* largest host batch (device staging)     */
    int32_t device;                 /* CUDA device ordinal                     */
    int32_t flags;                  /* enum vr_spec_flags                      */
} vr_agg_spec;

/* ---- batches ----------------------------------------------------------- */
enum vr_location { VR_HOST = 0, VR_DEVICE = 1 };

/* The strings a VR_DICT32 column's ids point into (an Arrow dictionary:
 * `size` entries, offsets[size + 1] into `data`, optional entry validity;
 * a null entry makes its rows null, GroupKeyTable.java:1388-1389). The struct
 * itself is in host memory; its buffers live where the batch lives.
 * `hashes` (optional) are the entries' HashKernels.hashBytes values
 * (NULL_MARK 0x7F4A7C15 for a null entry), e.g. from vr_hash_dictionary; a
 * caller that reuses one dictionary across batches computes them once. */
typedef struct vr_dictionary {
    int32_t size;
    int32_t reserved;
    const int32_t* offsets;
    const uint8_t* data;
    const uint8_t* validity;   /* NULL = every entry valid                  */
    const uint32_t* hashes;    /* NULL = computed where needed              */
} vr_dictionary;

typedef struct vr_column {
    const void* data;          /* values; VR_UTF8: the UTF-8 bytes          */
    const uint8_t* validity;   /* NULL = all valid                          */
    const int32_t* offsets;    /* VR_UTF8: n + 1 offsets into data          */
    const vr_dictionary* dictionary; /* VR_DICT32: the batch's dictionary;
                                  NULL = the ids are the spec's own (the
                                  caller keeps one dictionary for every batch) */
} vr_column;

typedef struct vr_batch {
    int64_t num_rows;
    const vr_column* columns;  /* spec->num_columns entries                    */
    const uint8_t* selection;  /* NULL = every row; unselected rows never
                                  create a group (GroupKeyTable.java:705-708)   */
    int32_t location;          /* enum vr_location                             */
    int32_t reserved;
} vr_batch;

typedef struct vr_out_column {
    void* data;
    uint8_t* validity;         /* ceil(n/8) bytes; written for every row       */
} vr_out_column;

typedef struct vr_agg_stats {
    int32_t tier;              /* 0 direct, 1 shared+global, 2 global           */
    int32_t warp_agg;          /* 1 when __match_any_sync pre-aggregation is on */
    int64_t table_capacity;    /* global slots                                  */
    int64_t slot_bytes;
    int64_t groups;            /* after the last sync                           */
    int64_t rows;              /* rows consumed                                 */
    int64_t batches;
    int64_t rehashes;
    int64_t deferred_rows;     /* rows replayed after a table grow              */
    int32_t threads;           /* per block                                     */
    int32_t blocks;            /* per launch                                    */
    int32_t smem_bytes;
    int32_t tile_rows;
    double last_kernel_ms;     /* VR_SPEC_TRACE only                            */
    double total_kernel_ms;
    double total_h2d_ms;
    double total_d2h_ms;
    int64_t kernel_launches;   /* every kernel this handle launched             */
    int32_t jit;               /* 1: the aggregate kernel was compiled for this spec */
    int32_t reserved;
} vr_agg_stats;

typedef struct vr_agg vr_agg;

/* ---- lifecycle ----------------------------------------------------------
 * vr_agg_create: GroupKeyTable + GroupedAggState construction
 *   (VectorAggFunction.newGroupedState, VectorAggregates.scala:100-111;
 *    GroupKeyTable constructor, GroupKeyTable.java:563-600). Returns
 *   VR_ERR_UNSUPPORTED for specs outside the GPU gate. */
int vr_agg_create(const vr_agg_spec* spec, vr_agg** out);

/* vr_agg_update: GroupKeyTable.assign + GroupedAggState.update for one batch
 *   (GroupKeyTable.java:709-764; VectorAggregates.scala:54-55;
 *    VectorHashAggregateExec.scala:584-602). Asynchronous on the handle's
 *   stream; host inputs are copied to HBM first. */
int vr_agg_update(vr_agg* h, const vr_batch* batch);

/* Waits for every queued update; surfaces device-side errors. */
int vr_agg_sync(vr_agg* h);

/* GroupKeyTable.size() (GroupKeyTable.java:683, the value assign returns at :709-764). Syncs. */
int vr_agg_num_groups(vr_agg* h, int64_t* groups);

/* Output columns: the keys, then each function's Spark buffer slots
 *   (VectorAggFunction.bufferTypes / emittedTypes, VectorAggregates.scala:100-111). */
int vr_agg_output_schema(const vr_agg* h, int32_t* num_out, vr_column_type* types, int32_t cap);

/* vr_agg_emit: groups [from, to) as Arrow columns into caller buffers
 *   (GroupKeyTable.writeKeys GroupKeyTable.java:2851-2920;
 *    GroupedAggState.writeBuffer VectorAggregates.scala:62, 179-198, 374-389;
 *    VectorGroupedAggregateIterator.buildBatch VectorHashAggregateExec.scala:831-913).
 *   Group order is the table's slot order (stable until the next update).
 *   `location` says where the output buffers live. */
int vr_agg_emit(vr_agg* h, int64_t from, int64_t to, const vr_out_column* outs, int32_t location);

/* Empties the table, keeping its memory (EmitAndReset,
 *   VectorHashAggregateExec.scala:193-246). A batch still in flight is
 *   settled first; the clear itself is queued on the handle's stream, ahead
 *   of later updates and emits, and does not wait for the device. */
int vr_agg_reset(vr_agg* h);

/* After vr_agg_emit returned VR_ERR_DECIMAL_PRECISION: the value that left
 * its type (unscaled, lo and hi limbs) and that type, which Spark's
 * NUMERIC_VALUE_OUT_OF_RANGE message names
 * (VectorErrors.decimalPrecisionOverflow, VectorErrors.scala:71-73).
 * VR_ERR_STATE when the emission recorded none (a total past 128 bits, or
 * a product row past its precision). */
int vr_agg_error_value(const vr_agg* h, int64_t* lo, int64_t* hi, int32_t* precision, int32_t* scale);

/* The table dictionary of key `key` (a VR_COL_BATCH_DICTIONARY key): the
 * strings its emitted table ids stand for, in id order (GroupKeyTable's
 * StringDictionary, GroupKeyTable.java:1308-1430; writeKeys emits them,
 * :2851-2920). Writes *size; with `offsets` (size + 1 entries) and `data`
 * (data_cap bytes) also the strings as an Arrow string array. *data_bytes
 * receives the bytes needed. Host memory; no device work. */
int vr_agg_key_dictionary(const vr_agg* h, int32_t key, int32_t* size, int32_t* offsets, uint8_t* data,
                          int64_t data_cap, int64_t* data_bytes);

/* Frees device state (GroupedAggState.close, VectorAggregates.scala:85-90). */
void vr_agg_destroy(vr_agg* h);

int vr_agg_get_stats(const vr_agg* h, vr_agg_stats* stats);
int vr_agg_last_error(const vr_agg* h, char* buf, size_t cap);
const char* vr_status_string(int status);
/* The message of the last failed vr_agg_create / vr_srv_* on this thread. */
const char* vr_thread_last_error(void);
/* The CUDA stream the handle launches on (cudaStream_t), for event timing. */
void* vr_agg_stream(const vr_agg* h);

/* ---- pinned host memory (the GPU analogue of NativePool, NativePool.java:76-87) */
int vr_host_alloc(size_t bytes, void** out);
int vr_host_free(void* p);
int vr_host_register(void* p, size_t bytes);
int vr_host_unregister(void* p);

/* ---- row hash parity (HashKernels.init/mixColumn/finish,
 *      kernels/.../HashKernels.java:42-236). Device pointers; out[n]. ------
 * Bit for bit the reference's row hash for every lane: INT32, INT64/FLOAT64
 * (folded), BOOL, DECIMAL128 (Decimal128.hash, folded), VR_UTF8
 * (HashKernels.hashBytes of each row's bytes, mixUtf8 :199-213) and
 * VR_DICT32 (hashBytes of each row's dictionary entry, mixDictionary
 * :215-236: the column must carry its dictionary). A null row mixes
 * NULL_MARK. Synchronous: returns once out_device is written. */
int vr_hash_rows(int32_t num_keys, const vr_column_type* types, const vr_column* keys,
                 int64_t num_rows, uint32_t* out_device, int32_t finish, void* stream);
/* HashKernels.hashBytes (HashKernels.java:183-197) of every entry of a
 * device-resident dictionary (NULL_MARK for a null entry) into
 * out_device[dict->size]; enqueued on `stream`, no allocation. */
int vr_hash_dictionary(const vr_dictionary* dict, uint32_t* out_device, void* stream);
/* vr_hash_rows without any device allocation, for callers that must not
 * allocate (a serving thread whose cudaMalloc/cudaFree would synchronise the
 * device under other queries, an executor at its memory cap). No counterpart
 * in the reference, whose hashing runs on the JVM heap. The key descriptors go
 * to a fixed 640-byte device scratch inside the library: at most 16 key
 * columns, more is VR_ERR_INVALID. A VR_DICT32 key must bring its
 * dictionary's entry hashes (dictionary->hashes, device memory, e.g. from
 * vr_hash_dictionary into the caller's buffer): computing them here would
 * need a buffer of the dictionary's size. An id outside the dictionary is not
 * reported (the call does not wait): such a row mixes 0 in that column.
 * Enqueues on `stream` and returns without waiting. Calls on one stream are ordered; calls that overlap in time on
 * other streams or threads share the scratch and race. The first call on a
 * device looks the scratch up and keeps its address for the life of the
 * process: a device reset (cudaDeviceReset) is not supported afterwards.
 * Do not capture this call into a CUDA graph: it copies the descriptors
 * from the caller's host arrays with cudaMemcpyAsync, and a captured copy
 * would read those arrays again at every replay, after they may be gone. */
int vr_hash_rows_noalloc(int32_t num_keys, const vr_column_type* types, const vr_column* keys,
                         int64_t num_rows, uint32_t* out_device, int32_t finish, void* stream);

/* ---- batched persistent aggregation ------------------------------------
 * Many independent instances (Spark tasks' batches) in one persistent
 * launch, optionally replayed from a CUDA graph. No reference analogue:
 * the reference runs one task per thread (VectorHashAggregateExec.scala:248-302).
 * The instances share one spec shape (one kernel) and one tier; the
 * persistent launch runs them all with one block shape and tile size, and
 * keeps each instance's own shared-memory strategy (its handle's tuner or
 * default choice): a shared-memory table that holds every group, a hot-key
 * cache in front of its HBM table, or its HBM table alone. VR_BATCHED_PLAIN
 * runs one launch per instance with each handle's own configuration. */
enum vr_batched_mode { VR_BATCHED_PERSISTENT = 0, VR_BATCHED_PLAIN = 1 };

typedef struct vr_tune_choice vr_tune_choice;

typedef struct vr_batched_plan {
    int32_t num_instances;
    vr_agg* const* instances;  /* handles created on the same device          */
    const vr_batch* batches;   /* one device-resident batch per instance     */
    int32_t mode;              /* enum vr_batched_mode                        */
    int32_t use_graph;         /* capture once, replay on later calls         */
    const vr_tune_choice* shape; /* persistent launch: consumer threads, tile
                                  rows, CTAs per SM and the hot-key cache slots
                                  (each 0 = default); NULL = every default    */
} vr_batched_plan;

typedef struct vr_batched_info {
    int32_t threads;           /* consumer threads per block                   */
    int32_t tile_rows;
    int32_t stages;
    int32_t blocks;            /* per launch                                   */
    int32_t smem_bytes;        /* dynamic shared memory per block              */
    int32_t smem_slots_max;    /* slots of the shared-memory area              */
    int32_t whole_tables;      /* instances with every group in shared memory  */
    int32_t caches;            /* instances with a hot-key cache before HBM    */
    int32_t hbm_only;          /* instances probing HBM directly               */
    int32_t jit;               /* 1: a kernel compiled for this spec and shape */
    int64_t total_tiles;
    int64_t total_rows;
    int64_t table_bytes;       /* HBM tables cleared by each run               */
} vr_batched_info;

typedef struct vr_batched vr_batched;
int vr_batched_create(const vr_batched_plan* plan, vr_batched** out);
/* Resets every instance's table, then aggregates every instance's batch. */
int vr_batched_run(vr_batched* b, void* stream);
int vr_batched_get_info(const vr_batched* b, vr_batched_info* info);
/* The autotuner for the persistent launch: instances grouped by the power of
 * two of their estimated groups, each group's shared-memory strategy (a
 * whole table, a 256/512/1,024-slot hot-key cache, or HBM alone) chosen by
 * coordinate descent on the launch's device time (`iters` timed runs per
 * candidate, the largest groups by rows first). The chosen strategies stay in
 * the plan and are recorded in the tuner's table (vr_tune_lookup) for each
 * instance's (spec, rows, estimated groups) bucket; *best_ms is the launch's
 * time with them. Runs the launch many times: every instance's table holds
 * the last run's groups afterwards. */
int vr_batched_tune(vr_batched* b, int32_t iters, double* best_ms);
void vr_batched_destroy(vr_batched* b);

/* ---- autotuner (table size, block shape, tier) keyed on rows and
 *      estimated cardinality ------------------------------------------- */
struct vr_tune_choice {
    int32_t tier;           /* 0 direct, 1 shared cache + HBM, 2 HBM only           */
    int32_t warp_agg;       /* __match_any_sync pre-aggregation                     */
    int32_t threads;        /* consumer threads per block (0 = default)             */
    int32_t blocks_per_sm;  /* 0 = default                                          */
    int32_t tile_rows;      /* rows per staged tile, multiple of 128 (0 = default)  */
    int32_t smem_slots;     /* shared cache slots, power of two (0 = default)       */
    int64_t table_capacity; /* HBM slots, power of two (0 = from est_groups)        */
};
/* vr_agg_create with a forced configuration (tests, the tuner's search). */
int vr_agg_create_tuned(const vr_agg_spec* spec, const vr_tune_choice* choice, vr_agg** out);
/* Runs every candidate configuration on one device-resident batch, times it
 * with CUDA events and records the fastest for (spec, rows, est_groups). */
int vr_tune_search(const vr_agg_spec* spec, const vr_batch* device_batch, int32_t iters, vr_tune_choice* best,
                   double* best_rows_per_s);

/* ---- plan inspection (host only; no GPU needed) ------------------------ */
typedef struct vr_plan_info {
    int32_t key_words;      /* packed key words per slot                           */
    int32_t acc_words;      /* accumulator words per slot                          */
    int32_t slot_words;
    int32_t num_ops;
    int32_t num_outputs;
    int32_t staged_columns;
    int32_t sentinel_layout;/* single 64-bit key stored xor a constant             */
    int32_t direct_ok;      /* dictionary / boolean keys: dense combination space  */
    int64_t direct_slots;
    char reason[160];       /* why a spec was refused                              */
} vr_plan_info;
int vr_agg_plan(const vr_agg_spec* spec, vr_plan_info* info, vr_column_type* out_types, int32_t cap);

/* Compiles the spec's specialised aggregate kernel for `tier` (0 direct,
 * 1 hash) with NVRTC -- host only, no GPU needed -- and reports the cubin
 * size; `log` receives the compiler log: the error on failure, ptxas's
 * resource usage (registers, spills, local memory) on success. */
int vr_jit_compile(const vr_agg_spec* spec, int32_t tier, int64_t* cubin_bytes, char* log, size_t cap);
/* The same for a given block shape: `threads` consumer threads (plus the
 * producer warp) and `min_blocks` CTAs per SM, the launch bounds that cap
 * the kernel's registers. */
int vr_jit_compile_shape(const vr_agg_spec* spec, int32_t tier, int32_t threads, int32_t min_blocks,
                         int64_t* cubin_bytes, char* log, size_t cap);
/* 1 and the recorded choice when the tuner has one for (spec, rows), else 0. */
int vr_tune_lookup(const vr_agg_spec* spec, int64_t rows, vr_tune_choice* out);
int vr_tune_record(const vr_agg_spec* spec, int64_t rows, const vr_tune_choice* choice, double rows_per_s);
int vr_tune_load(const char* path);
int vr_tune_save(const char* path);

/* ---- serving: continuous batching over resident per-query tables ------- */
typedef struct vr_srv_config {
    int32_t device;
    int32_t slots;             /* concurrent requests on the device           */
    int64_t hbm_cap_bytes;     /* admission cap for staging + tables          */
    int64_t staging_bytes_per_slot;
    int32_t flags;
    int32_t reserved;
} vr_srv_config;

typedef struct vr_srv_stats {
    int64_t submitted;
    int64_t completed;
    int64_t admitted_immediately;
    int64_t queued;            /* waited for a slot or for memory              */
    int64_t rejected;
    int64_t rows;
    double p50_ms;             /* submit -> result ready                       */
    double p99_ms;
    double max_ms;
    double mean_ms;
    int64_t hbm_in_use;
    int64_t hbm_peak;
    double p99_wait_ms;        /* submit -> admitted to the device             */
    double p99_service_ms;     /* admitted -> result ready                     */
    int64_t max_in_flight;     /* most requests admitted to the device and not
                                  yet complete at one time (> 1: requests of
                                  different queries overlapped on the device) */
} vr_srv_stats;

typedef struct vr_srv vr_srv;
int vr_srv_create(const vr_srv_config* cfg, vr_srv** out);
/* Opens a live query whose table stays resident in HBM. */
int vr_srv_open_query(vr_srv* s, const vr_agg_spec* spec, int32_t* query_id);
/* Queues one partial-aggregation batch (host memory, pinned for overlap).
 * The caller keeps the batch's buffers alive until the ticket completes. */
int vr_srv_submit(vr_srv* s, int32_t query_id, const vr_batch* batch, uint64_t* ticket);
/* Waits for a ticket; latency is submit -> device completion. */
int vr_srv_wait(vr_srv* s, uint64_t ticket, double* latency_ms);
/* Waits for every queued request of the query, then exposes its handle
 * for vr_agg_num_groups / vr_agg_emit. The server keeps ownership. */
int vr_srv_query_handle(vr_srv* s, int32_t query_id, vr_agg** h);
int vr_srv_close_query(vr_srv* s, int32_t query_id);
int vr_srv_get_stats(vr_srv* s, vr_srv_stats* st);
int vr_srv_drain(vr_srv* s);
void vr_srv_destroy(vr_srv* s);

/* ---- Parquet data pages -> Arrow columns on the device -------------------
 * The scan that feeds the aggregate: a column chunk's data pages, already
 * decompressed into device memory, decoded into one Arrow column without a
 * trip through host memory. Replaces ParquetPageDecoder.decode
 * (parquet/src/main/java/io/vecruntime/parquet/codec/ParquetPageDecoder.java:214-266)
 * with RleBitPackingReader (RleBitPackingReader.java:117-392) for the
 * definition levels and the dictionary ids, for flat columns (no repetition
 * levels). An RLE_DICTIONARY page decodes to its dictionary ids (int32), not
 * to resolved values: the column goes to the aggregate as VR_DICT32 with the
 * chunk's dictionary attached as a batch dictionary (VR_COL_BATCH_DICTIONARY;
 * vr_pq_plain_dictionary decodes a BYTE_ARRAY dictionary page into one), and
 * the aggregate maps each dictionary onto its table's once per batch. A
 * PLAIN page of a fixed-width type decodes to its values, a null slot
 * holding 0 (the reference leaves it unspecified). */
enum vr_pq_encoding { VR_PQ_PLAIN = 0, VR_PQ_RLE_DICTIONARY = 1 };

typedef struct vr_pq_page {
    const uint8_t* data;    /* device: the decompressed page. v1: [int32 LE byte length of
                               the levels][levels][values]; v2: [levels][values]; without
                               definition levels (max_def_level 0) only the values. RLE_DICTIONARY
                               values: one byte of id bit width, then the id stream */
    int64_t length;         /* bytes of the page */
    int32_t num_values;     /* slots in the page (one definition level each) */
    int32_t max_def_level;  /* a slot is present when its level equals this; 0: all present */
    int32_t v2;             /* data page v2: the levels' byte length is levels_length */
    int32_t levels_length;  /* v2 only */
    int32_t encoding;       /* enum vr_pq_encoding; every page of one call has the same */
    int32_t value_bytes;    /* PLAIN: 4 (INT32, FLOAT) or 8 (INT64, DOUBLE); RLE_DICTIONARY: 4 */
} vr_pq_page;

typedef struct vr_pq_decoder vr_pq_decoder;
/* A decoder on `device` for calls of up to `max_values` slots and
 * `max_bytes` page bytes in total (it sizes its device scratch for them).
 * One thread at a time per decoder; a call waits for the decoder's previous
 * call before it reuses its scratch. */
int vr_pq_create(int32_t device, int64_t max_values, int64_t max_bytes, vr_pq_decoder** out);
/* Decodes `num_pages` pages of one column chunk, in order, into one column
 * of the pages' slots in order: out_data (device; value_bytes per slot) and
 * out_validity (device, LSB-first bitmap, ceil(slots / 8) bytes; may be
 * NULL when no page has definition levels). Asynchronous on `stream` (a
 * cudaStream_t; NULL = the decoder's own). `pages` is read before the call
 * returns. A malformed page (a run header or payload past its stream, an
 * id stream with fewer ids than present slots, a bit width above 32) is
 * reported by vr_pq_sync. */
int vr_pq_decode(vr_pq_decoder* d, int32_t num_pages, const vr_pq_page* pages, void* out_data,
                 uint8_t* out_validity, void* stream);
/* Waits for the last decode; `present` (may be NULL) receives its count of
 * present slots. VR_ERR_INVALID for a malformed page, the page and the
 * reason in vr_thread_last_error (as for every vr_pq_* error). */
int vr_pq_sync(vr_pq_decoder* d, int64_t* present);
void vr_pq_destroy(vr_pq_decoder* d);
/* Host: a PLAIN-encoded BYTE_ARRAY dictionary page (num_values entries of an
 * int32 LE length and the bytes) into vr_dictionary buffers: offsets
 * (num_values + 1 int32) and data (*data_bytes bytes). With data == NULL it
 * only sets *data_bytes. Replaces ParquetPageDecoder.decodeDictionary
 * (ParquetPageDecoder.java:440-513) for BYTE_ARRAY. */
int vr_pq_plain_dictionary(const uint8_t* page, int64_t length, int32_t num_values, int32_t* offsets,
                           uint8_t* data, int64_t* data_bytes);

#ifdef __cplusplus
}
#endif
#endif /* VRGPU_H */
