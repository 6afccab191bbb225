/*
 * oracle.h -- CPU restatement of the reference's grouped aggregate.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for libvrgpu and the timed
 * CPU baseline. Nothing in the product path may call it.
 *
 * Restates, from the reference (vecruntime, Java / Scala):
 *   HashKernels (row hash)            kernels/src/main/java/io/vecruntime/kernels/HashKernels.java:42-236
 *   GroupKeyTable (general probe)     kernels/src/main/java/io/vecruntime/kernels/GroupKeyTable.java:709-764,
 *                                     2296-2371 (lookupOrInsert/equals), 2515-2561 (insert), 2631-2660 (rehash)
 *   GroupedAccumulators               kernels/src/main/java/io/vecruntime/kernels/GroupedAccumulators.java
 *   AggKernels / CompareOp NaN rules  AggKernels.java:40-41, 446-522; CompareOp.java:68-81
 *   Spark buffer rules                spark/src/main/scala/io/vecruntime/spark/agg/VectorAggregates.scala
 *   Parquet page decoding (pq_oracle.cpp)
 *                                     parquet/src/main/java/io/vecruntime/parquet/codec/RleBitPackingReader.java,
 *                                     ParquetPageDecoder.java:214-311, 415-497
 * It shares only the ABI structs (vrgpu.h) with the product; its table,
 * hashing and accumulators are its own code.
 */
#ifndef VR_ORACLE_H
#define VR_ORACLE_H

#include "vrgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_agg orc_agg;

enum orc_fp_mode {
    ORC_FP_SEQUENTIAL = 0,  /* the reference's strict order: sum += x per group, rows in order */
    ORC_FP_COMPENSATED = 1  /* Neumaier-compensated sums: the tolerance anchor for FP64 parity  */
};

int orc_agg_create(const vr_agg_spec* spec, orc_agg** out);
/* Host batch; processed in chunks of `chunk_rows` (the reference's batch
 * size, 4096 in VectorGroupedAggregateIterator; 0 = whole batch). */
int orc_agg_update(orc_agg* a, const vr_batch* batch, int64_t chunk_rows);
int64_t orc_agg_num_groups(const orc_agg* a);
int orc_agg_num_outputs(const orc_agg* a);
int orc_agg_output_type(const orc_agg* a, int i, vr_column_type* t);
/* Groups [from, to) in first-seen order into host buffers. */
int orc_agg_emit(orc_agg* a, int64_t from, int64_t to, const vr_out_column* outs, int fp_mode);
/* Folds every group of `src` into `dst` (the final merge of thread partials). */
int orc_agg_merge(orc_agg* dst, const orc_agg* src);
void orc_agg_destroy(orc_agg* a);
const char* orc_last_error(void);

/* Reference row hash (HashKernels.init/mixColumn, optional finish). */
int orc_hash_rows(int32_t num_keys, const vr_column_type* types, const vr_column* keys, int64_t n, uint32_t* out,
                  int32_t finish);

/* CPU baseline: rows split into `threads` contiguous partitions (one Spark
 * task each), each aggregated in `chunk_rows` batches into its own table,
 * then merged. Returns wall seconds in *seconds and the groups in *groups. */
int orc_agg_run_threads(const vr_agg_spec* spec, const vr_batch* batch, int32_t threads, int64_t chunk_rows,
                        double* seconds, int64_t* groups);

/* The strings behind key `key`'s emitted table ids (VR_COL_BATCH_DICTIONARY
 * keys), as vr_agg_key_dictionary returns them. */
int orc_agg_key_dictionary(const orc_agg* a, int32_t key, int32_t* size, int32_t* offsets, uint8_t* data,
                           int64_t data_cap, int64_t* data_bytes);

/* The same partitioned run folded into `dst` (the full-size parity check:
 * every group of the batch, ready for orc_agg_emit). */
int orc_agg_update_threads(orc_agg* dst, const vr_batch* batch, int32_t threads, int64_t chunk_rows);

/* Parquet pages (pq_oracle.cpp): RleBitPackingReader.readInts of n values
 * from a fresh reader, and ParquetPageDecoder.decode of one flat page into
 * ids / values and validity as vr_pq_decode writes them. */
int orc_rle_decode(const uint8_t* buf, int64_t len, int32_t bit_width, int64_t n, uint32_t* out);
int orc_pq_decode_page(const uint8_t* page, const vr_pq_page* desc, void* out_data, uint8_t* out_validity,
                       int64_t* present_count);
int orc_pq_plain_dictionary(const uint8_t* page, int64_t length, int32_t num_values, int32_t* offsets,
                            uint8_t* data, int64_t* data_bytes);
const char* orc_pq_last_error(void);
/* Many pages of one chunk on `threads` host threads (the timed CPU
 * baseline), each page into its own output: slots at slot_base[k], validity
 * bytes at valid_base[k]. */
int orc_pq_decode_pages_threads(int32_t num_pages, const uint8_t* const* pages, const vr_pq_page* descs,
                                const int64_t* slot_base, const int64_t* valid_base, void* out_data,
                                uint8_t* out_validity, int32_t threads, double* seconds);

#ifdef __cplusplus
}
#endif
#endif
