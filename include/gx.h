/*
 * gx.h — C ABI of the B200-native relational operator core.
 *
 * Every entry point takes plain pointers, sizes and enums (no C++ or torch
 * types), returns a gx_status, and reports a human-readable message through
 * gx_last_error_message() when the status is not GX_OK.  Device memory in
 * views is caller-owned; device memory in results (gx_table / gx_column) is
 * owned by this library's stream-ordered pool and released with
 * gx_table_free / gx_free.
 *
 * Reference interface that each entry point replaces is cited beside it as
 * path:line inside the reference project (src/cuda/...).  The C++ header
 * include/gamax/gamax.hpp rebuilds the reference's exact gamax:: signatures
 * on top of these functions.
 */
#ifndef GX_H_
#define GX_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t without pulling in the CUDA headers. */
typedef struct CUstream_st* gx_stream_t;

/* ---------------------------------------------------------------------- */
/* Types — same enumerator order as gamax::type_id                         */
/* (src/cuda/types/data_type.hpp:12-28).                                   */
/* ---------------------------------------------------------------------- */
typedef enum gx_type_id {
    GX_EMPTY = 0,
    GX_INT8 = 1,
    GX_INT16 = 2,
    GX_INT32 = 3,
    GX_INT64 = 4,
    GX_BOOL8 = 5,
    GX_UINT8 = 6,
    GX_UINT16 = 7,
    GX_UINT32 = 8,
    GX_UINT64 = 9,
    GX_FLOAT32 = 10,
    GX_FLOAT64 = 11,
    GX_STRING = 12,
    GX_NUM_TYPE_IDS = 13
} gx_type_id;

typedef enum gx_status {
    GX_OK = 0,
    GX_EINVAL = 1,       /* std::runtime_error in the reference: bad shape/type/hint */
    GX_ENOMEM = 2,       /* std::bad_alloc in the reference */
    GX_ECUDA = 3,        /* a CUDA runtime call failed */
    GX_EOVERFLOW = 4,    /* a capacity (table, output buffer, batch) was exceeded */
    GX_ETIMEOUT = 5,     /* a bounded device-side wait gave up */
    GX_EUNSUPPORTED = 6  /* valid request this library does not implement */
} gx_status;

typedef enum gx_sort_order { GX_ASCENDING = 0, GX_DESCENDING = 1 } gx_sort_order;

/*
 * Column view: mirrors gamax::column_view{data, size, type, offset}
 * (src/cuda/memory/column.hpp:13-94).  `size` is the number of visible rows
 * and element i lives at (char*)data + (offset + i) * size_of(type).
 * For GX_STRING the view's `data` points to a gx_string_columns struct in
 * host memory holding device pointers (ARROW layout: chars + int64 offsets
 * of length rows+1; the view's offset skips rows of the offsets array,
 * src/cuda/string/string_column.hpp:22-90).
 */
typedef struct gx_column_view {
    void* data;
    int64_t size;
    int32_t type;
    int64_t offset;
} gx_column_view;

typedef struct gx_string_columns {
    const char* chars;      /* device */
    const int64_t* offsets; /* device, rows+1 entries */
} gx_string_columns;

/* gamax::table_view (src/cuda/memory/table.hpp:76-150). */
typedef struct gx_table_view {
    const gx_column_view* columns; /* host array of num_columns views */
    int64_t num_columns;
} gx_table_view;

/* An owned device column handed to the caller (free with gx_free).  A
 * released GX_STRING column's buffer holds its size+1 int64 offsets
 * followed by the characters (ARROW layout); the view of a STRING column
 * still inside a gx_table points to a gx_string_columns owned by the table. */
typedef struct gx_column {
    void* data;             /* device; NULL when size == 0 */
    int64_t size;           /* rows */
    int32_t type;
    int64_t capacity_bytes; /* allocation size; may exceed size*sizeof(type) */
} gx_column;

/* Owned result table (gamax::table, src/cuda/memory/table.hpp:152-225). */
typedef struct gx_table gx_table;

int64_t gx_table_num_columns(const gx_table* t);
int64_t gx_table_num_rows(const gx_table* t);
/* Non-owning view of column i. */
gx_status gx_table_column(const gx_table* t, int64_t i, gx_column_view* out);
/* Moves column i out of the table (the slot becomes empty, indices keep). */
gx_status gx_table_release_column(gx_table* t, int64_t i, gx_column* out);
void gx_table_free(gx_table* t);

/* Stream-ordered pool allocator (replaces allocate_mem/release_mem,
 * src/cuda/memory/mem_manager.hpp:118-159). */
gx_status gx_malloc(void** ptr, size_t bytes, gx_stream_t stream);
gx_status gx_free(void* ptr, gx_stream_t stream);
/* Current and peak pool bytes handed out by gx_malloc and internal
 * allocations (MemoryManager::get_mem_used / peak,
 * src/cuda/memory/mem_manager.hpp:12-29). */
gx_status gx_mem_stats(int64_t* current_bytes, int64_t* peak_bytes);
gx_status gx_mem_reset_peak(void);

/* Copies between host and device (cudaMemcpyAsync + stream sync). */
gx_status gx_copy(void* dst, const void* src, size_t bytes, gx_stream_t stream);
gx_status gx_stream_sync(gx_stream_t stream);

/* Last error message of the calling thread (never NULL). */
const char* gx_last_error_message(void);
/* Library version string. */
const char* gx_version(void);
/* Number of kernels this library has launched in this process. */
int64_t gx_kernel_launch_count(void);
/* Per-kernel timing with CUDA events recorded on the launching stream
 * around each named hot kernel (e.g. "hash_groupby", "join_probe_write").
 * gx_profile_read synchronises on the recorded events and returns the
 * summed milliseconds and the number of launches since the last reset. */
void gx_profile_enable(int32_t on);
gx_status gx_profile_read(const char* kernel, double* total_ms, int64_t* launches);
void gx_profile_reset(void);

/* ---------------------------------------------------------------------- */
/* Group-by — gamax::groupby (src/cuda/operators/groupby/groupby.hpp:16-49,*/
/* src/cuda/operators/groupby/aggregation.hpp:8-30).                      */
/* ---------------------------------------------------------------------- */
typedef enum gx_agg_kind {
    GX_AGG_SUM = 0,
    GX_AGG_MAX = 1,
    GX_AGG_MIN = 2,
    GX_AGG_AVG = 3,
    GX_AGG_ANY = 4,
    GX_AGG_COUNT_ALL = 5
} gx_agg_kind;

typedef struct gx_agg_request {
    int64_t column_index; /* ignored for COUNT_ALL */
    int32_t agg_kind;     /* gx_agg_kind */
} gx_agg_request;

/* Same enumerator order as gamax::groupby::groupby_algo
 * (src/cuda/operators/groupby/groupby.hpp:16-25). */
typedef enum gx_groupby_algo {
    GX_GB_AUTO = 0,
    GX_GB_HASH = 1,
    GX_GB_SORT = 2,
    GX_GB_SORT_OPT = 3,
    GX_GB_SORT_GFUR = 4,
    GX_GB_PARTITION = 5,
    GX_GB_PARTITION_GFUR = 6,
    GX_GB_UNSUPPORTED = 7
} gx_groupby_algo;

/* Strategy used when groupby_algo == GX_GB_AUTO. */
typedef enum gx_selector_kind {
    GX_SELECT_HEURISTIC = 0, /* the reference's NDV threshold rule (groupby.cu:68-119) */
    GX_SELECT_LEARNED = 1    /* the FP16 MLP loaded with gx_selector_load */
} gx_selector_kind;

/*
 * groupby_hint (src/cuda/operators/groupby/groupby.hpp:27-42) plus three
 * extension fields.  It is in/out exactly like the reference's non-const
 * reference: AUTO writes the chosen algorithm into groupby_algo and
 * SORT_OPT sets optimize_sort.
 */
typedef struct gx_groupby_hint {
    int64_t groups_upper_bound; /* INT64_MAX = unknown */
    int32_t zero_based_ids;
    int32_t optimize_sort;
    int32_t groupby_algo;       /* gx_groupby_algo */
    int32_t agg_count;
    int32_t enable_skf;
    int32_t allow_hash_fallback;
    /* extensions */
    int32_t selector;           /* gx_selector_kind, used by AUTO */
    int32_t radix_bits;         /* partition fan-out log2 (0 = engine picks); out: bits used */
    int32_t load_factor_pct;    /* hash table fill target in percent (0 = engine picks) */
    int32_t reserved;
} gx_groupby_hint;

/* Fills a hint with the reference's defaults. */
void gx_groupby_hint_init(gx_groupby_hint* hint);

/*
 * Grouped aggregation over one key column.
 * Output table: [key, one column per request in request order,
 * + COUNT column when hint->agg_count], with the reference's output types
 * (agg_output_data_type, src/cuda/operators/groupby/aggregate.cu:41-53).
 * Replaces gamax::groupby::groupby (groupby.cu:396-465).
 */
gx_status gx_groupby(const gx_table_view* key, const gx_table_view* val,
                     const gx_agg_request* requests, int32_t num_requests,
                     gx_groupby_hint* hint, gx_stream_t stream, gx_table** out);

/* Variant entry points: gamax::groupby::hash::groupby (groupby_hash.hpp:17-22),
 * sort::groupby / sort::groupby_gfur (groupby_sort.hpp:17-29),
 * partition::groupby / partition::groupby_gfur (groupby_partition.hpp:52-64). */
gx_status gx_groupby_hash(const gx_table_view* key, const gx_table_view* val,
                          const gx_agg_request* requests, int32_t num_requests,
                          gx_groupby_hint* hint, gx_stream_t stream, gx_table** out);
gx_status gx_groupby_sort(const gx_table_view* key, const gx_table_view* val,
                          const gx_agg_request* requests, int32_t num_requests,
                          gx_groupby_hint* hint, gx_stream_t stream, gx_table** out);
gx_status gx_groupby_sort_gfur(const gx_table_view* key, const gx_table_view* val,
                               const gx_agg_request* requests, int32_t num_requests,
                               gx_groupby_hint* hint, gx_stream_t stream, gx_table** out);
gx_status gx_groupby_partition(const gx_table_view* key, const gx_table_view* val,
                               const gx_agg_request* requests, int32_t num_requests,
                               gx_groupby_hint* hint, gx_stream_t stream, gx_table** out);
gx_status gx_groupby_partition_gfur(const gx_table_view* key, const gx_table_view* val,
                                    const gx_agg_request* requests, int32_t num_requests,
                                    gx_groupby_hint* hint, gx_stream_t stream,
                                    gx_table** out);

/* hash::distinct / sort::distinct (groupby_hash.hpp:24-34, groupby_sort.hpp:31-47):
 * one row per distinct key. */
gx_status gx_distinct_hash(const gx_table_view* key, gx_groupby_hint* hint,
                           gx_stream_t stream, gx_table** out);
gx_status gx_distinct_sort(const gx_table_view* key, gx_groupby_hint* hint,
                           gx_stream_t stream, gx_table** out);

/* Scalar aggregate over a whole table: groupby::aggregate::aggregate
 * (aggregation.hpp:32-37, aggregate.cu:55-). One-row result. */
gx_status gx_aggregate(const gx_table_view* input, const gx_agg_request* requests,
                       int32_t num_requests, gx_stream_t stream, gx_table** out);

/* Output type of an aggregation (agg_output_data_type, aggregate.cu:41-53). */
int32_t gx_agg_output_type(int32_t agg_kind, int32_t input_type);

/* Key tables that are not one numeric column: gx_groupby / gx_distinct_*
 * accept STRING keys and several key columns (the reference hashes whole
 * rows, groupby_hash.cu:437-498).  With hint->enable_skf integral key
 * columns are first packed into one 64-bit key (smart key fusion,
 * groupby.cu:403-465); the output holds the original key columns, gathered
 * at one row of each group, then the aggregates. */

/* Smart key fusion: packs integral key columns into one UINT64 column, each
 * column taking (value - min) on ceil(log2(range + 1)) bits, or its
 * dictionary code when that is narrower and the range saves fewer than 2/3
 * of the column's bits; equal packed keys <=> equal key rows.  Returns
 * GX_EUNSUPPORTED (the reference returns nullptr) when a column is not
 * integral or the key needs more than max_bits bits; *total_bits gets the
 * bits used.  Replaces compress::multikey_compress
 * (compress/multikey_compress.hpp:29-32, multikey_compress.cu:25-399). */
gx_status gx_multikey_compress(const gx_table_view* key, int32_t max_bits, gx_stream_t stream,
                               gx_column* out, int32_t* total_bits);

/* out[i] = input[gather_map[i]] for numeric or STRING columns (INT64 row
 * ids).  Replaces util::device::gather (utils/transform.hpp, transform.cu:168-186)
 * and the string gather of join materialisation (join/materialize.cu:26-30). */
gx_status gx_gather(gx_column_view gather_map, gx_column_view input, gx_stream_t stream, gx_column* out);

/* ---------------------------------------------------------------------- */
/* Filter — gamax::select (src/cuda/operators/select/select.hpp:15-64) and  */
/* the mask utilities of gamax::util::device (src/cuda/utils/transform.hpp: */
/* 34-48).  A predicate list compares columns with literals and combines    */
/* the comparisons with AND or OR (the reference evaluates general          */
/* expression trees, expr/expr_fast.hpp; those are not part of this ABI).   */
/* Masks are BOOL8 columns, one byte per row (nonzero = keep).             */
/* ---------------------------------------------------------------------- */
typedef enum gx_cmp_op {
    GX_CMP_LT = 0, GX_CMP_LE = 1, GX_CMP_GT = 2, GX_CMP_GE = 3, GX_CMP_EQ = 4, GX_CMP_NE = 5,
    GX_CMP_BETWEEN = 6 /* lo <= x < hi */
} gx_cmp_op;
typedef enum gx_combine { GX_COMBINE_AND = 0, GX_COMBINE_OR = 1 } gx_combine;

/* column (op) literal.  Integer columns compare with lo_i / hi_i (as
 * uint64 bits for unsigned columns), float columns with lo_f / hi_f. */
typedef struct gx_predicate {
    int64_t column_index;
    int32_t op;        /* gx_cmp_op */
    int32_t reserved;
    int64_t lo_i, hi_i;
    double lo_f, hi_f;
} gx_predicate;

/* BOOL8 mask of the rows the predicates keep (select_to_bitmask,
 * select.hpp:30-34).  1 to 8 predicates on numeric columns. */
gx_status gx_select_to_bitmask(const gx_table_view* table, const gx_predicate* predicates,
                               int32_t num_predicates, int32_t combine, gx_stream_t stream,
                               gx_column* mask);
/* The kept rows of every column, in input order; the predicates are
 * evaluated while compacting, so no mask is written (select with
 * fuse_operations, select.hpp:15-24). */
gx_status gx_select(const gx_table_view* table, const gx_predicate* predicates,
                    int32_t num_predicates, int32_t combine, gx_stream_t stream, gx_table** out);
/* Rows of every (numeric) column whose mask byte is nonzero, in input order
 * (util::device::compact(table_view, mask), transform.hpp:34-48). */
gx_status gx_compact(const gx_table_view* input, gx_column_view mask, gx_stream_t stream,
                     gx_table** out);
/* Rows whose value is not zero (util::device::count_nonzero). */
gx_status gx_count_nonzero(gx_column_view column, gx_stream_t stream, int64_t* count);

/* ---------------------------------------------------------------------- */
/* Inner equi-join — gamax::join (src/cuda/operators/join/join.hpp:7-33,   */
/* inner_join.hpp:11-15).                                                 */
/* ---------------------------------------------------------------------- */
typedef enum gx_join_algo {
    GX_JOIN_AUTO = 0, GX_JOIN_HASH = 1, GX_JOIN_SORT = 2, GX_JOIN_PARTITION = 3,
    GX_JOIN_UNSUPPORTED = 4
} gx_join_algo;
typedef enum gx_mat_algo {
    GX_MAT_AUTO = 0, GX_MAT_GFUR = 1, GX_MAT_GFTR = 2, GX_MAT_INDEX_CLUSTER = 3,
    GX_MAT_UNSUPPORTED = 4
} gx_mat_algo;

/* How the SORT join matches once the inputs are ordered. */
typedef enum gx_join_sort_mode {
    GX_JOIN_SORTED_BUILD = 0, /* sort the smaller side, probe the other in place */
    GX_JOIN_SORT_MERGE = 1    /* sort both sides, then merge-path match */
} gx_join_sort_mode;

#define GX_MAX_JOIN_OUTPUT_SIZE (((int64_t)1) << 30)

typedef struct gx_join_hint {
    int32_t sorted_left;
    int32_t sorted_right;
    int32_t unique_left;
    int32_t unique_right;
    int64_t max_out;   /* 0 = no limit */
    int32_t join_algo; /* gx_join_algo */
    int32_t mat_algo;  /* gx_mat_algo */
    /* extension */
    int32_t sort_mode; /* gx_join_sort_mode */
    int32_t reserved;
} gx_join_hint;

void gx_join_hint_init(gx_join_hint* hint);

/*
 * Inner equi-join on column 0 of each side.  Output:
 * [key, left payloads..., right payloads...] with one row per matching
 * (left row, right row) pair.  Replaces gamax::join::inner_eq_join
 * (inner_join.cu:206-229) for algo SORT (GFTR and GFUR).
 */
gx_status gx_inner_eq_join(const gx_table_view* left, const gx_table_view* right,
                           const gx_join_hint* hint, gx_stream_t stream, gx_table** out);

/* Join returning matched row-id pairs only: out columns [left_rowid, right_rowid]
 * (int64), the index form used by GFUR materialisation
 * (sort_merge_join.cu:249-293). */
gx_status gx_inner_eq_join_rowids(gx_column_view left_key, gx_column_view right_key,
                                  const gx_join_hint* hint, gx_stream_t stream,
                                  gx_table** out);

/* ---------------------------------------------------------------------- */
/* Radix sort — gamax::sort (src/cuda/operators/sort/sort.hpp:14-75).       */
/* A stable LSD radix sort on bits [begin_bit, end_bit) of the order-       */
/* preserving key image; end_bit <= 0 means the full key width.            */
/* d_temp / temp_bytes: optional caller scratch (gx_sort_temp_bytes).       */
/* ---------------------------------------------------------------------- */
gx_status gx_sort_temp_bytes(int64_t num_rows, int32_t key_type, int32_t val_type,
                             size_t* temp_bytes);
gx_status gx_sort_column_pair(gx_column_view key, gx_column_view val, int32_t begin_bit,
                              int32_t end_bit, int32_t order, void* d_temp,
                              size_t temp_bytes, gx_stream_t stream, gx_column* key_out,
                              gx_column* val_out);
gx_status gx_sort_column(gx_column_view col, int32_t begin_bit, int32_t end_bit,
                         int32_t order, void* d_temp, size_t temp_bytes,
                         gx_stream_t stream, gx_column* out);
/* argsort: (sorted keys, int64 source row ids). */
gx_status gx_argsort(gx_column_view col, int32_t begin_bit, int32_t end_bit, int32_t order,
                     void* d_temp, size_t temp_bytes, gx_stream_t stream,
                     gx_column* key_out, gx_column* idx_out);
/* gx_sort_column_pair without any memory allocation; no counterpart in the
 * reference.  Same stable sort, same result, written into caller device
 * buffers key_out / val_out (size*width bytes each, overlapping neither
 * each other nor the inputs).  For callers that cannot allocate: an engine
 * whose buffer manager owns all of device memory, or one that cannot take
 * the device synchronisation an allocation may cause.  Temporaries come from
 * one fixed 8 MiB array in device memory: keys and values 4 or 8 bytes wide,
 * and a sort needing more scratch (about 0.5 M pairs of 8+8 bytes) fails
 * with GX_EINVAL before any launch.  No scratch byte has to start at zero.
 * All calls on a device share the array, so calls that overlap on the
 * device race; order them on one stream or with events.  The first call on
 * a device looks up the array's address (cudaGetSymbolAddress, which may
 * load device code) and sets the scatter kernel's shared-memory attribute
 * for every 4/8-byte width pair: make it before any stream capture begins.
 * Later calls, of any width pair, only launch kernels and queue copies.
 * Returns without waiting for the sort to finish. */
gx_status gx_sort_column_pair_noalloc(gx_column_view key, gx_column_view val, int32_t begin_bit,
                                      int32_t end_bit, int32_t order, void* key_out,
                                      void* val_out, gx_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Radix partition — gamax::partition                                      */
/* (src/cuda/operators/partition/partition.hpp:11-79).  A partition is a    */
/* stable reorder by bits [begin_bit, end_bit).                             */
/* ---------------------------------------------------------------------- */
gx_status gx_partition_column_pair(gx_column_view key, gx_column_view val,
                                   int32_t begin_bit, int32_t end_bit, void* d_temp,
                                   size_t temp_bytes, gx_stream_t stream,
                                   gx_column* key_out, gx_column* val_out);
gx_status gx_partition_column(gx_column_view col, int32_t begin_bit, int32_t end_bit,
                              void* d_temp, size_t temp_bytes, gx_stream_t stream,
                              gx_column* out);
gx_status gx_arg_partition(gx_column_view col, int32_t begin_bit, int32_t end_bit,
                           void* d_temp, size_t temp_bytes, gx_stream_t stream,
                           gx_column* key_out, gx_column* idx_out);
/* Inclusive offsets of the 2^(end-begin) partitions of an already
 * partitioned column: out[p] = rows with digit <= p; out has 2^(end-begin)+1
 * int64 entries and the last one equals the row count
 * (compute_partition_offsets, partition.cu:122-171). */
gx_status gx_compute_partition_offsets(gx_column_view partitioned_key, int32_t begin_bit,
                                       int32_t end_bit, gx_stream_t stream,
                                       gx_column* out);

/* ---------------------------------------------------------------------- */
/* Dictionary encoding — gamax::compress                                   */
/* (src/cuda/compress/dictionary_encode.hpp:12-37).                        */
/* ---------------------------------------------------------------------- */
/* Hash encode: dense codes in [0, NDV) (dictionary_encode.cu:144-225). */
gx_status gx_dictionary_encode(gx_column_view col, int32_t encode_type,
                               int64_t dictionary_size_hint, double load_factor,
                               gx_stream_t stream, gx_column* out, int64_t* dict_size);
/* Order-preserving encode: code = rank among distinct values
 * (dictionary_encode.cu:228-334). */
gx_status gx_dictionary_encode_with_order(gx_column_view col, int32_t encode_type,
                                          int64_t dictionary_size_hint,
                                          double load_factor, gx_stream_t stream,
                                          gx_column* out, int64_t* dict_size);
/* Encode against a ready dictionary: code = position of the value in
 * `dict`; a value absent from it gets INT32_MIN
 * (dictionary_encode_dict_ready.cu:16-82).  INT32 codes only. */
gx_status gx_dictionary_encode_with_dict(gx_column_view col, gx_column_view dict,
                                         int32_t encode_type, gx_stream_t stream,
                                         gx_column* out);
/* String hash encode over an ARROW string column (a GX_STRING view): int32
 * codes dense in [0, NDV), in first-insert order like the numeric hash
 * encode; *dict_size = NDV.  The reference's dictionary_encode rejects
 * STRING (dictionary_encode.cu:32-34); this is its string counterpart. */
gx_status gx_dictionary_encode_strings(gx_column_view col, int64_t dictionary_size_hint,
                                       gx_stream_t stream, gx_column* codes,
                                       int64_t* dict_size);

/* ---------------------------------------------------------------------- */
/* Statistics — gamax::stats (src/cuda/stats/stats_compute.hpp:60-80).      */
/* ---------------------------------------------------------------------- */
/* HyperLogLog distinct-count estimate, 2^13 registers (standard error
 * about 1.15%, the reference's sd 0.0122197, stats_compute.cu:103-153). */
gx_status gx_compute_ndv_approx(gx_column_view col, gx_stream_t stream, int64_t* ndv);
/* min / max of an integer or float column, widened to int64 / double bits. */
gx_status gx_compute_min_max(gx_column_view col, gx_stream_t stream, void* min_out,
                             void* max_out);

/* ---------------------------------------------------------------------- */
/* Synthetic data generators (seeded, counter-based; identical on CPU).     */
/* ---------------------------------------------------------------------- */
typedef enum gx_key_dist {
    GX_DIST_UNIFORM = 0,  /* iid uniform rank in [0, G) */
    GX_DIST_CYCLIC = 1,   /* rank = bijective_shuffle(i) mod G: exactly N/G per key */
    GX_DIST_ZIPF = 2,     /* P(rank r) ∝ 1/(r+1)^s via inverse CDF */
    GX_DIST_SEQUENCE = 3, /* rank = i */
    GX_DIST_ZIPF_APPROX = 4 /* Zipf by the closed-form inverse of the continuous
                               CDF, no table; device only (training data) */
} gx_key_dist;

typedef struct gx_gen_spec {
    uint64_t seed;
    uint64_t stream_id;   /* independent sub-stream */
    int32_t dist;         /* gx_key_dist */
    int32_t scatter;      /* 1: key = bijective_mix(rank) instead of rank */
    int64_t groups;       /* G */
    double zipf_s;
    const double* zipf_cdf; /* device CDF from gx_zipf_cdf (dist == ZIPF) */
    int64_t lo, hi;       /* value range [lo, hi) for integer value columns */
    double miss_frac;     /* keys: this fraction draws rank G + uniform[0, G) instead */
} gx_gen_spec;

/* Zipf CDF over G ranks, computed on the host in double and uploaded:
 * cdf[r] = sum_{j<=r} (j+1)^-s / total, cdf[G-1] = 1. */
gx_status gx_zipf_cdf_host(int64_t groups, double s, double* cdf_host);
/* Fill a device column. Keys use dist/scatter/groups; integer value columns
 * draw uniform [lo, hi); FLOAT64/FLOAT32 draw uniform [0, 1). */
gx_status gx_generate_keys(gx_column_view out, const gx_gen_spec* spec, gx_stream_t stream);
gx_status gx_generate_values(gx_column_view out, const gx_gen_spec* spec, gx_stream_t stream);
/* Random permutation of [0, n) (n a power of two) plus `base` as int32/int64. */
gx_status gx_generate_permutation(gx_column_view out, uint64_t seed, int64_t base,
                                  gx_stream_t stream);
/* ARROW string column from dictionary codes: row i gets the bytes of
 * dictionary entry codes[i] (dict_chars / dict_offsets, device); out_offsets
 * (rows+1, device) must already hold the prefix sum of the row lengths. */
gx_status gx_generate_strings(const char* dict_chars, const int64_t* dict_offsets, int64_t dict_size,
                              const int32_t* codes, int64_t rows, const int64_t* out_offsets,
                              char* out_chars, gx_stream_t stream);
/* int64 sequence start, start+step, ... (make_sequence, column.cu:48-55). */
gx_status gx_fill_sequence(gx_column_view out, int64_t start, int64_t step,
                           gx_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Learned strategy selector.                                              */
/* ---------------------------------------------------------------------- */
#define GX_SEL_NUM_FEATURES 20   /* 16 key-sample features + 4 of the aggregation list */
#define GX_SEL_KEY_FEATURES 16
#define GX_SEL_HIDDEN 64
#define GX_SEL_NUM_VARIANTS 3   /* 0 = HASH, 1 = SORT, 2 = PARTITION */
#define GX_SEL_NUM_FANOUTS 4    /* radix bits {8, 10, 12, 14} */
#define GX_SEL_NUM_OUTPUTS (GX_SEL_NUM_VARIANTS + GX_SEL_NUM_FANOUTS)
#define GX_SEL_SAMPLE_ROWS 16384

/* Sketch of a 2^14-row strided sample of a key column: HLL distinct
 * estimate of the sample, top-8 key frequencies, rows/distinct ratio,
 * dtype and log-size terms: features 0..15 of GX_SEL_NUM_FEATURES floats
 * (16..19 are written as zero; see gx_selector_plan_features). */
gx_status gx_selector_features(gx_column_view key, gx_stream_t stream, float* features_host);
/* Features 16..19 (written to out4[0..3]): the aggregation list the group-by
 * will run — value bytes read per row / 32, accumulators / 8, float SUM
 * accumulators / 4, MIN and MAX accumulators / 8 — as AUTO sees them. */
gx_status gx_selector_plan_features(const gx_table_view* val, const gx_agg_request* requests,
                                    int32_t num_requests, int32_t agg_count, float* out4);
/* Number of fp16 parameters of the 3-layer MLP. */
int64_t gx_selector_param_count(void);
/* Install trained fp16 weights (host array of gx_selector_param_count halves). */
gx_status gx_selector_load(const uint16_t* params_fp16_host, const float* feat_mean,
                           const float* feat_std);
/* The request lists the loaded weights were trained on, as their plan
 * features (gx_selector_plan_features: 4 floats each, `count` lists): AUTO
 * with the learned selector runs the network only for a request list whose
 * plan features lie within `radius` (largest coordinate difference) of one
 * of them, and the plain NDV rule otherwise.  count = 0 (the state before
 * any call) trusts the network for every list.  Host only. */
gx_status gx_selector_set_plan_support(const float* plan_features_host, int32_t count, float radius);
/* Forward pass for a batch of feature rows on the device: writes
 * GX_SEL_NUM_OUTPUTS scores per row (lower is better). */
gx_status gx_selector_predict(const float* features_host, int32_t rows, float* scores_host);
/* Raw MLP kernels for training (all device pointers).
 * params: fp16 weights; x: [rows, F] fp32 standardised features;
 * target: [rows, OUT] fp32; mask: [rows, OUT] fp32 (1 = supervised);
 * grads: fp32 gradient of the masked mean squared error;
 * loss: fp32 scalar. */
gx_status gx_mlp_forward(const void* params_fp16, const float* x, int32_t rows, float* out,
                         gx_stream_t stream);
gx_status gx_mlp_forward_backward(const void* params_fp16, const float* x,
                                  const float* target, const float* mask, int32_t rows,
                                  float* grads, float* loss, gx_stream_t stream);
/* Adam step on fp32 master weights, re-emitting fp16 weights. */
gx_status gx_mlp_adam_step(float* master, void* params_fp16, const float* grads, float* m,
                           float* v, int32_t step, float lr, gx_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Batched engine: many uneven group-by pipelines in one launch.           */
/* Each instance: dictionary-encode an ARROW string key column, keep rows  */
/* with lo <= date < hi, group by the encoded key with SUM(int64) and      */
/* COUNT.  Output per instance: dictionary strings in code order and the   */
/* per-code SUM / COUNT.                                                   */
/* ---------------------------------------------------------------------- */
typedef struct gx_batch_instance {
    const char* chars;        /* device, string key column (ARROW) */
    const int64_t* offsets;   /* device, rows+1 */
    const int32_t* date;      /* device, rows */
    const int64_t* amount;    /* device, rows, fixed-point decimal (scale 2) */
    int64_t rows;
    int32_t date_lo, date_hi; /* keep lo <= date < hi */
} gx_batch_instance;

typedef struct gx_batch_result {
    int64_t num_groups;       /* distinct strings among kept rows */
    int64_t* sum;             /* device, capacity >= dict capacity */
    int64_t* count;           /* device */
    int64_t* first_row;       /* device: a row holding the group's string */
} gx_batch_result;

typedef struct gx_batch_plan gx_batch_plan;

/* Plan a batch: validates the descriptors, runs the autotuner (tile rows,
 * table load factor) and sizes per-instance tables.  `max_distinct` bounds
 * the dictionary of every instance (gx_batch_run encodes the strings of the
 * rows its date range keeps; the per-instance engine encodes every row). */
gx_status gx_batch_plan_create(const gx_batch_instance* instances, int32_t count,
                               int64_t max_distinct, gx_stream_t stream,
                               gx_batch_plan** plan);
/* One persistent launch over all instances (captured once into a CUDA graph,
 * replayed on later calls). */
gx_status gx_batch_run(gx_batch_plan* plan, gx_stream_t stream);
/* The same work as one launch sequence per instance (the plain engine). */
gx_status gx_batch_run_per_instance(gx_batch_plan* plan, gx_stream_t stream);
gx_status gx_batch_results(const gx_batch_plan* plan, gx_batch_result* results_host);
/* Tile rows and load factor the autotuner chose. */
gx_status gx_batch_tuning(const gx_batch_plan* plan, int32_t* tile_rows,
                          int32_t* load_factor_pct);
void gx_batch_plan_free(gx_batch_plan* plan);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* GX_H_ */
