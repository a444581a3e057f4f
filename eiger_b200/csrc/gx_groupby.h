// gx_groupby.h — internal interfaces between the operator translation units.
#pragma once

#include "gx_agg.cuh"

namespace gx {

// ----- hash group-by (gx_groupby_hash.cu) -----
void init_records(uint64_t* recs, int64_t nrec, const agg_desc& d, uint64_t empty, cudaStream_t s);
int hash_smem_slots(const agg_desc& d, int key_width, int64_t groups_bound, int* replicas);
// Sample sketch of a key column (gx_selector.cu): f[6..13] are the shares of
// the 8 most frequent keys in a 2^14-row strided sample.
void selector_features(const col& key, float* f, cudaStream_t s);
// A work unit of radix-partitioned rows: rows [begin, end) of one partition;
// split = the partition is spread over several units.
struct part_unit {
    int64_t begin, end;
    int split, pad;
};
// Aggregates partitioned rows unit by unit in shared-memory tables (the hash
// group-by's table code); `shift` = partition bits of the key hash, gpp =
// expected groups per partition.  Final groups of whole, unspilled units are
// appended to orec / *ocount; the rest merge into the global record table
// grec (gcap records + the sentinel record; gflags[0] sentinel, [1] overflow).
// Returns false when the groups per partition do not fit a shared table.
// dense_only: only the dense-id kernel (false when the plan has no compiled
// form or its tables do not fit).
bool hash_units_aggregate(const void* keys, int kw, int kind, const agg_desc& d, const part_unit* units,
                          const int64_t* n_units, int64_t gpp, int shift, uint64_t* grec, uint64_t gcap, int* gflags,
                          uint64_t* orec, unsigned long long* ocount, int64_t rec_cap, int* rec_ovf, cudaStream_t s,
                          bool dense_only = false);
void hash_groupby(const col& key, const agg_plan& p, gx_groupby_hint* hint, cudaStream_t s,
                  gx_table* out);

// ----- sort / partition group-by (gx_groupby_sort.cu, gx_groupby_partition.cu) -----
void sort_groupby(const col& key, const agg_plan& p, gx_groupby_hint* hint, bool gfur,
                  cudaStream_t s, gx_table* out);
void partition_groupby(const col& key, const agg_plan& p, gx_groupby_hint* hint, bool gfur,
                       cudaStream_t s, gx_table* out);

// Radix-partitions (key, row id) by R bits of the partition hash; see
// gx_groupby_partition.cu.
void hash_partition_rows(const col& key, int R, void* keys_out, int64_t* rows_out, int64_t* part_start,
                         cudaStream_t s);

// ----- radix sort / partition (gx_radix.cu) -----
// Stable LSD radix sort of (key, value) on bits [begin_bit, end_bit) of the
// order-preserving key image.  vals_in may be null (keys only) or, with
// vals_iota, the values are the row ids 0..n-1 (int64).  Outputs are
// caller-allocated.  Key types: any numeric; value widths 4 or 8 (or 0).
struct radix_temp {
    dbuf own;
    void* ptr = nullptr;
    size_t bytes = 0;
};
size_t radix_temp_bytes(int64_t n, int key_width, int val_width);
void radix_sort(const col& keys, const void* vals_in, int val_width, bool vals_iota,
                int begin_bit, int end_bit, bool descending, void* keys_out, void* vals_out,
                void* temp, size_t temp_bytes, cudaStream_t s);
// Pair sort (4/8-byte keys and values) with all temporaries carved from
// caller scratch of radix_pairs_scratch_bytes(n, kw, vw) bytes.
size_t radix_pairs_scratch_bytes(int64_t n, int key_width, int val_width);
void radix_sort_pairs_scratch(const col& keys, const void* vals_in, int val_width, int begin_bit, int end_bit,
                              bool descending, void* keys_out, void* vals_out, char* scratch, cudaStream_t s);
// Sets, on the current device, the kernel attributes every 4/8-byte pair
// scatter needs (each is otherwise set before its first launch).
void radix_prepare_pair_scatters();
// Key image width in bits for a type (the default end_bit).
inline int key_bits(int type) { return 8 * size_of(type); }

// Min/max of the order-preserving image (for trimming radix passes).
void key_image_range(const col& keys, uint64_t* lo, uint64_t* hi, cudaStream_t s);
// One stable radix-sort digit pass through the partition plan's bulk-copy
// scatter (gx_groupby_partition.cu); false when it does not apply.
bool radix_pass_bulk(const void* kin, const void* vin, int kw, int vw, bool iota, int64_t n, const img_params& ip,
                     int shift, int dbits, int tile_rows, const int64_t* offs, void* kout, void* vout, int* err,
                     cudaStream_t s);

// ----- statistics (gx_hll.cu) -----
int64_t ndv_estimate(const col& key, cudaStream_t s);
// Min / max of a numeric column, widened to int64 (integers) or double
// bits (floats) (gx_hll.cu).
void compute_min_max(const col& key, void* min_out, void* max_out, cudaStream_t s);

// ----- dictionary encoding (gx_dict.cu, gx_batch.cu) -----
// mode 0: hash codes (first-insert order), 1: order-preserving codes.
void dictionary_encode(const gx_column_view& v, int encode_type, int64_t size_hint, double load_factor, int mode,
                       cudaStream_t s, gx_column* out, int64_t* dict_size);
// ARROW string column -> int32 codes dense in [0, NDV).
void dictionary_encode_strings(const gx_column_view& v, int64_t size_hint, cudaStream_t s, gx_column* out,
                               int64_t* ndv);

// ----- keys that are not one numeric column (gx_keys.cu) -----
// One int64 / uint64 key per row that is equal exactly when all key
// columns are equal.  With `skf`, integral columns are bit-packed by value
// range (the reference's smart key fusion); otherwise, or when packing
// does not fit 64 bits, columns are dictionary-encoded and chained.
// *groups_bound gets an upper bound of the distinct keys.
owned_col derive_group_key(const gx_table_view* key, bool skf, cudaStream_t s, int64_t* groups_bound);
// Bit-packs integral key columns by value range into one UINT64 column
// (src/cuda/compress/multikey_compress.cu:25-399); returns false when a
// column is not integral or the packed key needs more than max_bits.
bool multikey_compress(const gx_table_view* key, int max_bits, cudaStream_t s, owned_col* out, int* total_bits);
// ----- filter (gx_select.cu) -----
void select_to_bitmask(const gx_table_view* t, const gx_predicate* preds, int n, int combine, cudaStream_t s,
                       gx_column* mask);
void select_rows(const gx_table_view* t, const gx_predicate* preds, int n, int combine, cudaStream_t s,
                 gx_table* out);
void compact_by_mask(const gx_table_view* t, const gx_column_view& mask, cudaStream_t s, gx_table* out);
int64_t count_nonzero(const gx_column_view& v, cudaStream_t s);

// out = column v gathered at row ids idx[0..n) (numeric or STRING).
owned_col gather_column(const gx_column_view& v, const int64_t* idx, int64_t n, cudaStream_t s);

}  // namespace gx
