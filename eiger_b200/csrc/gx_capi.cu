// gx_capi.cu — the extern "C" boundary.  Every entry point converts C
// views into internal columns, runs the operator, and maps exceptions to a
// gx_status plus a thread-local message (the reference throws
// std::runtime_error / std::bad_alloc; include/gamax/gamax.hpp maps the
// status back to those exception types).
#include <cstdlib>
#include <cstring>
#include <new>

#include "gx_groupby.h"

namespace gx {
void groupby_dispatch(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req, int nreq,
                      gx_groupby_hint* hint, int forced_algo, cudaStream_t s, gx_table* out);
void distinct_dispatch(const gx_table_view* key, gx_groupby_hint* hint, int algo, cudaStream_t s, gx_table* out);
void aggregate_dispatch(const gx_table_view* input, const gx_agg_request* req, int nreq, cudaStream_t s,
                        gx_table* out);
void inner_eq_join(const gx_table_view* left, const gx_table_view* right, const gx_join_hint* hint,
                   cudaStream_t s, gx_table* out);
void inner_eq_join_rowids(const gx_column_view& l, const gx_column_view& r, const gx_join_hint* hint,
                          cudaStream_t s, gx_table* out);
void dictionary_encode(const gx_column_view& v, int encode_type, int64_t size_hint, double load_factor, int mode,
                       cudaStream_t s, gx_column* out, int64_t* dict_size);
void dictionary_encode_with_dict(const gx_column_view& v, const gx_column_view& dv, int encode_type, cudaStream_t s,
                                 gx_column* out);
void compute_min_max(const col& key, void* min_out, void* max_out, cudaStream_t s);
void zipf_cdf_host(int64_t G, double s, double* cdf);
void generate_keys(const gx_column_view& v, const gx_gen_spec& sp, cudaStream_t s);
void generate_values(const gx_column_view& v, const gx_gen_spec& sp, cudaStream_t s);
void generate_permutation(const gx_column_view& v, uint64_t seed, int64_t base_v, cudaStream_t s);
void radix_sort_biased(const col& keys_c, const void* vals_in, int val_width, bool vals_iota, int begin_bit,
                       int end_bit, bool descending, uint64_t bias, void* keys_out, void* vals_out, void* temp,
                       size_t temp_bytes, cudaStream_t s);
void generate_strings(const char* dchars, const int64_t* doff, int64_t dsize, const int32_t* codes, int64_t rows,
                      const int64_t* off, char* out, cudaStream_t s);
void selector_features(const col& key, float* f, cudaStream_t s);
void selector_plan_features(const agg_plan& p, float* f4);
int64_t selector_param_count();
void selector_load(const uint16_t* params, const float* mean, const float* stdv);
void selector_set_plan_support(const float* f4, int count, float radius);
void selector_predict(const float* feats, int rows, float* scores, cudaStream_t s);
void mlp_forward(const void* params, const float* x, int rows, float* out, cudaStream_t s);
void mlp_forward_backward(const void* params, const float* x, const float* tgt, const float* mask, int rows,
                          float* grads, float* loss, cudaStream_t s);
void mlp_adam(float* master, void* params, const float* grads, float* m, float* v, int step, float lr,
              cudaStream_t s);
}  // namespace gx

namespace {
thread_local std::string t_err;

gx_status set_err(gx_status s, const char* msg) {
    t_err = msg ? msg : "";
    return s;
}
}  // namespace

#define GX_TRY(...)                                                   \
    try {                                                             \
        t_err.clear();                                                \
        __VA_ARGS__;                                                  \
        return GX_OK;                                                 \
    } catch (const gx::error& e) {                                    \
        return set_err(e.status, e.what());                           \
    } catch (const std::bad_alloc& e) {                               \
        return set_err(GX_ENOMEM, e.what());                          \
    } catch (const std::exception& e) {                               \
        return set_err(GX_EINVAL, e.what());                          \
    }

using gx::col;
using gx::resolve;

static cudaStream_t cs(gx_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

namespace gx {
void set_last_error(const char* msg) { t_err = msg ? msg : ""; }
}  // namespace gx

extern "C" {

const char* gx_last_error_message(void) { return t_err.c_str(); }
const char* gx_version(void) { return "gx 0.1 (sm_100a)"; }
int64_t gx_kernel_launch_count(void) { return gx::g_launches.load(); }
void gx_profile_enable(int32_t on) { gx::g_profiling.store(on ? 1 : 0); }
gx_status gx_profile_read(const char* kernel, double* total_ms, int64_t* launches) {
    GX_TRY({
        gx::require(kernel != nullptr, "null kernel name");
        gx::prof_read(kernel, total_ms, launches, false);
    })
}
void gx_profile_reset(void) { gx::prof_read("", nullptr, nullptr, true); }

int64_t gx_table_num_columns(const gx_table* t) { return t ? (int64_t)t->cols.size() : 0; }
int64_t gx_table_num_rows(const gx_table* t) {
    if (!t) return 0;
    for (auto& c : t->cols)
        if (c.present) return c.size;
    return 0;
}
gx_status gx_table_column(const gx_table* t, int64_t i, gx_column_view* out) {
    GX_TRY({
        gx::require(t && out, "null argument");
        gx::require(i >= 0 && i < (int64_t)t->cols.size(), "column out of range");
        gx::require(t->cols[i].present, "column was released");
        // A STRING column's view points to its host-side (chars, offsets) pair.
        out->data = t->cols[i].type == GX_STRING ? (void*)t->cols[i].str.get() : t->cols[i].buf.get();
        out->size = t->cols[i].size;
        out->type = t->cols[i].type;
        out->offset = 0;
    })
}
gx_status gx_table_release_column(gx_table* t, int64_t i, gx_column* out) {
    GX_TRY({
        gx::require(t && out, "null argument");
        gx::require(i >= 0 && i < (int64_t)t->cols.size(), "column out of range");
        gx::require(t->cols[i].present, "column was released");
        *out = gx::to_gx_column(std::move(t->cols[i]));
        t->cols[i].present = false;
    })
}
void gx_table_free(gx_table* t) { delete t; }

gx_status gx_malloc(void** ptr, size_t bytes, gx_stream_t s) {
    GX_TRY({
        gx::require(ptr != nullptr, "null argument");
        *ptr = bytes ? gx::pool_alloc(bytes, cs(s)) : nullptr;
    })
}
gx_status gx_free(void* ptr, gx_stream_t s) { GX_TRY({ gx::pool_free(ptr, cs(s)); }) }
gx_status gx_mem_stats(int64_t* cur, int64_t* peak) { GX_TRY({ gx::pool_stats(cur, peak); }) }
gx_status gx_mem_reset_peak(void) { GX_TRY({ gx::pool_reset_peak(); }) }
gx_status gx_copy(void* dst, const void* src, size_t bytes, gx_stream_t s) {
    GX_TRY({
        if (bytes) GX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, cs(s)));
        GX_CUDA(cudaStreamSynchronize(cs(s)));
    })
}
gx_status gx_stream_sync(gx_stream_t s) { GX_TRY({ GX_CUDA(cudaStreamSynchronize(cs(s))); }) }

void gx_groupby_hint_init(gx_groupby_hint* h) {
    if (!h) return;
    std::memset(h, 0, sizeof(*h));
    h->groups_upper_bound = INT64_MAX;
    h->groupby_algo = GX_GB_AUTO;
}
void gx_join_hint_init(gx_join_hint* h) {
    if (!h) return;
    std::memset(h, 0, sizeof(*h));
}

int32_t gx_agg_output_type(int32_t agg_kind, int32_t input_type) { return gx::agg_output_type(agg_kind, input_type); }

static gx_status run_groupby(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req, int32_t n,
                             gx_groupby_hint* hint, int algo, gx_stream_t s, gx_table** out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        *out = nullptr;
        std::unique_ptr<gx_table> t(new gx_table);
        gx::groupby_dispatch(key, val, req, n, hint, algo, cs(s), t.get());
        *out = t.release();
    })
}

gx_status gx_groupby(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req, int32_t n,
                     gx_groupby_hint* hint, gx_stream_t s, gx_table** out) {
    return run_groupby(key, val, req, n, hint, -1, s, out);
}
gx_status gx_groupby_hash(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req, int32_t n,
                          gx_groupby_hint* hint, gx_stream_t s, gx_table** out) {
    return run_groupby(key, val, req, n, hint, GX_GB_HASH, s, out);
}
gx_status gx_groupby_sort(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req, int32_t n,
                          gx_groupby_hint* hint, gx_stream_t s, gx_table** out) {
    return run_groupby(key, val, req, n, hint, hint && hint->optimize_sort ? GX_GB_SORT_OPT : GX_GB_SORT, s, out);
}
gx_status gx_groupby_sort_gfur(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req,
                               int32_t n, gx_groupby_hint* hint, gx_stream_t s, gx_table** out) {
    return run_groupby(key, val, req, n, hint, GX_GB_SORT_GFUR, s, out);
}
gx_status gx_groupby_partition(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req,
                               int32_t n, gx_groupby_hint* hint, gx_stream_t s, gx_table** out) {
    return run_groupby(key, val, req, n, hint, GX_GB_PARTITION, s, out);
}
gx_status gx_groupby_partition_gfur(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req,
                                    int32_t n, gx_groupby_hint* hint, gx_stream_t s, gx_table** out) {
    return run_groupby(key, val, req, n, hint, GX_GB_PARTITION_GFUR, s, out);
}

gx_status gx_distinct_hash(const gx_table_view* key, gx_groupby_hint* hint, gx_stream_t s, gx_table** out) {
    GX_TRY({
        gx::require(out && hint, "null argument");
        std::unique_ptr<gx_table> t(new gx_table);
        gx::distinct_dispatch(key, hint, GX_GB_HASH, cs(s), t.get());
        *out = t.release();
    })
}
gx_status gx_distinct_sort(const gx_table_view* key, gx_groupby_hint* hint, gx_stream_t s, gx_table** out) {
    GX_TRY({
        gx::require(out && hint, "null argument");
        std::unique_ptr<gx_table> t(new gx_table);
        gx::distinct_dispatch(key, hint, GX_GB_SORT, cs(s), t.get());
        *out = t.release();
    })
}
gx_status gx_aggregate(const gx_table_view* input, const gx_agg_request* req, int32_t n, gx_stream_t s,
                       gx_table** out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        std::unique_ptr<gx_table> t(new gx_table);
        gx::aggregate_dispatch(input, req, n, cs(s), t.get());
        *out = t.release();
    })
}

gx_status gx_select_to_bitmask(const gx_table_view* table, const gx_predicate* preds, int32_t n, int32_t combine,
                               gx_stream_t s, gx_column* mask) {
    GX_TRY({
        gx::require(mask != nullptr, "null output");
        gx::select_to_bitmask(table, preds, n, combine, cs(s), mask);
    })
}

gx_status gx_select(const gx_table_view* table, const gx_predicate* preds, int32_t n, int32_t combine, gx_stream_t s,
                    gx_table** out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        std::unique_ptr<gx_table> t(new gx_table);
        gx::select_rows(table, preds, n, combine, cs(s), t.get());
        *out = t.release();
    })
}

gx_status gx_compact(const gx_table_view* input, gx_column_view mask, gx_stream_t s, gx_table** out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        std::unique_ptr<gx_table> t(new gx_table);
        gx::compact_by_mask(input, mask, cs(s), t.get());
        *out = t.release();
    })
}

gx_status gx_count_nonzero(gx_column_view column, gx_stream_t s, int64_t* count) {
    GX_TRY({
        gx::require(count != nullptr, "null output");
        *count = gx::count_nonzero(column, cs(s));
    })
}

gx_status gx_multikey_compress(const gx_table_view* key, int32_t max_bits, gx_stream_t s, gx_column* out,
                               int32_t* total_bits) {
    GX_TRY({
        gx::require(key && out, "null argument");
        gx::require(max_bits >= 1 && max_bits <= 64, "multikey_compress: max_fused_key_bits must be in 1..64");
        gx::owned_col fused;
        int bits = 0;
        if (!gx::multikey_compress(key, max_bits, cs(s), &fused, &bits))
            gx::fail(GX_EUNSUPPORTED, "multikey_compress: keys are not all integral or need more than " +
                                          std::to_string(max_bits) + " bits");
        if (total_bits) *total_bits = bits;
        *out = gx::to_gx_column(std::move(fused));
    })
}

gx_status gx_gather(gx_column_view gather_map, gx_column_view input, gx_stream_t s, gx_column* out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        gx::require(gather_map.type == GX_INT64, "gather: the gather map must be INT64 row ids");
        col m = resolve(gather_map);
        gx::owned_col o = gx::gather_column(input, m.as<int64_t>(), m.n, cs(s));
        GX_CUDA(cudaStreamSynchronize(cs(s)));
        *out = gx::to_gx_column(std::move(o));
    })
}

gx_status gx_inner_eq_join(const gx_table_view* left, const gx_table_view* right, const gx_join_hint* hint,
                           gx_stream_t s, gx_table** out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        std::unique_ptr<gx_table> t(new gx_table);
        gx::inner_eq_join(left, right, hint, cs(s), t.get());
        *out = t.release();
    })
}
gx_status gx_inner_eq_join_rowids(gx_column_view l, gx_column_view r, const gx_join_hint* hint, gx_stream_t s,
                                  gx_table** out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        std::unique_ptr<gx_table> t(new gx_table);
        gx::inner_eq_join_rowids(l, r, hint, cs(s), t.get());
        *out = t.release();
    })
}

gx_status gx_sort_temp_bytes(int64_t n, int32_t key_type, int32_t val_type, size_t* temp_bytes) {
    GX_TRY({
        gx::require(temp_bytes != nullptr, "null output");
        *temp_bytes = gx::radix_temp_bytes(n, gx::size_of(key_type), val_type == GX_EMPTY ? 0 : 8);
    })
}

static void sort_common(gx_column_view key, const gx_column_view* val, bool iota, int32_t b, int32_t e,
                        int32_t order, void* d_temp, size_t temp_bytes, cudaStream_t s, gx_column* kout,
                        gx_column* vout) {
    col k = resolve(key);
    gx::require(gx::is_numeric(k.type), "sort: unsupported key type " + gx::type_name(k.type));
    gx::require(order == GX_ASCENDING || order == GX_DESCENDING, "sort: bad order");
    gx::owned_col ko = gx::make_col(k.type, k.n, s);
    gx::owned_col vo;
    const void* vin = nullptr;
    int vw = 0;
    gx::owned_col vwide;  // narrow values travel as row ids + gather
    bool gather_vals = false;
    col v;
    if (val) {
        v = resolve(*val);
        gx::require(v.n == k.n, "sort: key and value columns differ in length");
        gx::require(gx::is_numeric(v.type), "sort: unsupported value type");
        vo = gx::make_col(v.type, v.n, s);
        vw = gx::size_of(v.type);
        vin = v.data;
        if (vw < 4) gather_vals = true;
    } else if (iota) {
        vo = gx::make_col(GX_INT64, k.n, s);
        vw = 8;
    }
    if (gather_vals) {
        gx::dbuf idx((size_t)std::max<int64_t>(k.n, 1) * 8, s);
        gx::radix_sort_biased(k, nullptr, 8, true, b, e, order == GX_DESCENDING, 0, ko.buf.get(), idx.get(), d_temp,
                              temp_bytes, s);
        gx::gather_bytes(vo.buf.get(), v.data, idx.get<int64_t>(), k.n, vw, s);
    } else {
        gx::radix_sort_biased(k, vin, vw, iota, b, e, order == GX_DESCENDING, 0, ko.buf.get(),
                              vw ? vo.buf.get() : nullptr, d_temp, temp_bytes, s);
    }
    GX_CUDA(cudaStreamSynchronize(s));
    *kout = gx::to_gx_column(std::move(ko));
    if (vout) *vout = gx::to_gx_column(std::move(vo));
}

gx_status gx_sort_column_pair(gx_column_view key, gx_column_view val, int32_t b, int32_t e, int32_t order, void* d_temp,
                              size_t temp_bytes, gx_stream_t s, gx_column* kout, gx_column* vout) {
    GX_TRY({
        gx::require(kout && vout, "null output");
        sort_common(key, &val, false, b, e, order, d_temp, temp_bytes, cs(s), kout, vout);
    })
}
gx_status gx_sort_column(gx_column_view col_v, int32_t b, int32_t e, int32_t order, void* d_temp, size_t temp_bytes,
                         gx_stream_t s, gx_column* out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        sort_common(col_v, nullptr, false, b, e, order, d_temp, temp_bytes, cs(s), out, nullptr);
    })
}
gx_status gx_argsort(gx_column_view col_v, int32_t b, int32_t e, int32_t order, void* d_temp, size_t temp_bytes,
                     gx_stream_t s, gx_column* kout, gx_column* iout) {
    GX_TRY({
        gx::require(kout && iout, "null output");
        sort_common(col_v, nullptr, true, b, e, order, d_temp, temp_bytes, cs(s), kout, iout);
    })
}
gx_status gx_partition_column_pair(gx_column_view key, gx_column_view val, int32_t b, int32_t e, void* d_temp,
                                   size_t temp_bytes, gx_stream_t s, gx_column* kout, gx_column* vout) {
    return gx_sort_column_pair(key, val, b, e, GX_ASCENDING, d_temp, temp_bytes, s, kout, vout);
}
gx_status gx_partition_column(gx_column_view col_v, int32_t b, int32_t e, void* d_temp, size_t temp_bytes,
                              gx_stream_t s, gx_column* out) {
    return gx_sort_column(col_v, b, e, GX_ASCENDING, d_temp, temp_bytes, s, out);
}
gx_status gx_arg_partition(gx_column_view col_v, int32_t b, int32_t e, void* d_temp, size_t temp_bytes, gx_stream_t s,
                           gx_column* kout, gx_column* iout) {
    return gx_argsort(col_v, b, e, GX_ASCENDING, d_temp, temp_bytes, s, kout, iout);
}

}  // extern "C"

namespace gx {
namespace {
// Digit histogram of (key >> b) & mask on the raw value (RadixExtractor,
// src/cuda/operators/partition/partition.cu:103-120): a shared-memory
// histogram per block for up to 4096 digits, global atomics above that.
template <typename T>
__global__ void k_digit_hist(const T* __restrict__ keys, int64_t n, int b, uint64_t mask, int P,
                             unsigned long long* __restrict__ counts) {
    extern __shared__ unsigned long long sh[];
    const bool local = P <= 4096;
    if (local)
        for (int i = threadIdx.x; i < P; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t d = ((uint64_t)keys[i] >> b) & mask;
        atomicAdd(local ? &sh[d] : &counts[d], 1ull);
    }
    __syncthreads();
    if (local)
        for (int i = threadIdx.x; i < P; i += blockDim.x)
            if (sh[i]) atomicAdd(&counts[i], sh[i]);
}
}  // namespace
}  // namespace gx

extern "C" gx_status gx_compute_partition_offsets(gx_column_view key, int32_t b, int32_t e, gx_stream_t s,
                                                  gx_column* out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        col k = resolve(key);
        gx::require(gx::is_signed_int(k.type) || gx::is_unsigned_int(k.type),
                    "Cannot extract radix from non-integral type");
        gx::require(e > b && e - b <= 30, "partition offsets: bad bit range");
        // Inclusive offsets over the digit histogram, valid for any order of
        // the keys (HistogramEven + InclusiveSum, partition.cu:122-171):
        // out[p] = rows with digit <= p, out[P] = rows.
        int P = 1 << (e - b);
        gx::owned_col o = gx::make_col(GX_INT64, P + 1, cs(s));
        uint64_t mask = (uint64_t)P - 1;
        gx::dbuf counts((size_t)P * 8, cs(s)), ex((size_t)(P + 1) * 8, cs(s));
        gx::fill_u64(counts.get(), 0, P, cs(s));
        if (k.n > 0) {
            const int g = gx::grid_for(k.n, 256, 4);
            const size_t sh = P <= 4096 ? (size_t)P * 8 : 0;
            switch (gx::size_of(k.type)) {
                case 1: gx::k_digit_hist<<<g, 256, sh, cs(s)>>>(k.as<uint8_t>(), k.n, b, mask, P, counts.get<unsigned long long>()); break;
                case 2: gx::k_digit_hist<<<g, 256, sh, cs(s)>>>(k.as<uint16_t>(), k.n, b, mask, P, counts.get<unsigned long long>()); break;
                case 4: gx::k_digit_hist<<<g, 256, sh, cs(s)>>>(k.as<uint32_t>(), k.n, b, mask, P, counts.get<unsigned long long>()); break;
                default: gx::k_digit_hist<<<g, 256, sh, cs(s)>>>(k.as<uint64_t>(), k.n, b, mask, P, counts.get<unsigned long long>()); break;
            }
            GX_LAUNCHED();
        }
        gx::exclusive_scan_i64(counts.get<int64_t>(), ex.get<int64_t>(), P, cs(s));
        GX_CUDA(cudaMemcpyAsync(o.buf.get<int64_t>(), ex.get<int64_t>() + 1, (size_t)P * 8, cudaMemcpyDeviceToDevice, cs(s)));
        GX_CUDA(cudaMemcpyAsync(o.buf.get<int64_t>() + P, ex.get<int64_t>() + P, 8, cudaMemcpyDeviceToDevice, cs(s)));
        GX_CUDA(cudaStreamSynchronize(cs(s)));
        *out = gx::to_gx_column(std::move(o));
    })
}

extern "C" {

gx_status gx_dictionary_encode(gx_column_view c, int32_t et, int64_t hint, double lf, gx_stream_t s, gx_column* out,
                               int64_t* ds) {
    GX_TRY({
        gx::require(out && ds, "null output");
        gx::dictionary_encode(c, et, hint, lf, 0, cs(s), out, ds);
    })
}
gx_status gx_dictionary_encode_with_order(gx_column_view c, int32_t et, int64_t hint, double lf, gx_stream_t s,
                                          gx_column* out, int64_t* ds) {
    GX_TRY({
        gx::require(out && ds, "null output");
        gx::dictionary_encode(c, et, hint, lf, 1, cs(s), out, ds);
    })
}
gx_status gx_dictionary_encode_with_dict(gx_column_view c, gx_column_view d, int32_t et, gx_stream_t s,
                                         gx_column* out) {
    GX_TRY({
        gx::require(out != nullptr, "null output");
        gx::dictionary_encode_with_dict(c, d, et, cs(s), out);
    })
}

gx_status gx_compute_ndv_approx(gx_column_view c, gx_stream_t s, int64_t* ndv) {
    GX_TRY({
        gx::require(ndv != nullptr, "null output");
        col k = resolve(c);
        gx::require(gx::is_numeric(k.type), "ndv: unsupported column type " + gx::type_name(k.type));
        *ndv = gx::ndv_estimate(k, cs(s));
    })
}
gx_status gx_compute_min_max(gx_column_view c, gx_stream_t s, void* mn, void* mx) {
    GX_TRY({
        gx::require(mn && mx, "null output");
        gx::compute_min_max(resolve(c), mn, mx, cs(s));
    })
}

gx_status gx_selector_plan_features(const gx_table_view* val, const gx_agg_request* req, int32_t n, int32_t agg_count,
                                    float* out4) {
    GX_TRY({
        gx::require(out4 != nullptr, "null output");
        gx::selector_plan_features(gx::make_agg_plan(val, req, n, agg_count != 0), out4);
    })
}

gx_status gx_selector_features(gx_column_view key, gx_stream_t s, float* features) {
    GX_TRY({
        gx::require(features != nullptr, "null output");
        col k = resolve(key);
        gx::require(gx::is_numeric(k.type), "selector: numeric key column required");
        gx::selector_features(k, features, cs(s));
    })
}
int64_t gx_selector_param_count(void) { return gx::selector_param_count(); }
gx_status gx_selector_load(const uint16_t* params, const float* mean, const float* stdv) {
    GX_TRY({
        gx::require(params != nullptr, "null weights");
        gx::selector_load(params, mean, stdv);
    })
}
gx_status gx_selector_set_plan_support(const float* plan_features, int32_t count, float radius) {
    GX_TRY({
        gx::require(count >= 0 && (count == 0 || plan_features != nullptr), "bad plan support list");
        gx::require(radius >= 0.f, "negative support radius");
        gx::selector_set_plan_support(plan_features, count, radius);
    })
}
gx_status gx_selector_predict(const float* features, int32_t rows, float* scores) {
    GX_TRY({
        gx::require(features && scores && rows >= 0, "bad arguments");
        gx::selector_predict(features, rows, scores, nullptr);
    })
}
gx_status gx_mlp_forward(const void* params, const float* x, int32_t rows, float* out, gx_stream_t s) {
    GX_TRY({ gx::mlp_forward(params, x, rows, out, cs(s)); })
}
gx_status gx_mlp_forward_backward(const void* params, const float* x, const float* target, const float* mask,
                                  int32_t rows, float* grads, float* loss, gx_stream_t s) {
    GX_TRY({ gx::mlp_forward_backward(params, x, target, mask, rows, grads, loss, cs(s)); })
}
gx_status gx_mlp_adam_step(float* master, void* params, const float* grads, float* m, float* v, int32_t step,
                           float lr, gx_stream_t s) {
    GX_TRY({
        gx::require(step >= 1, "adam: step counts from 1");
        gx::mlp_adam(master, params, grads, m, v, step, lr, cs(s));
    })
}

gx_status gx_zipf_cdf_host(int64_t groups, double sk, double* cdf) {
    GX_TRY({
        gx::require(groups > 0 && cdf, "zipf: bad arguments");
        gx::zipf_cdf_host(groups, sk, cdf);
    })
}
gx_status gx_generate_keys(gx_column_view out, const gx_gen_spec* sp, gx_stream_t s) {
    GX_TRY({
        gx::require(sp != nullptr, "null spec");
        gx::generate_keys(out, *sp, cs(s));
        GX_CUDA(cudaStreamSynchronize(cs(s)));
    })
}
gx_status gx_generate_values(gx_column_view out, const gx_gen_spec* sp, gx_stream_t s) {
    GX_TRY({
        gx::require(sp != nullptr, "null spec");
        gx::generate_values(out, *sp, cs(s));
        GX_CUDA(cudaStreamSynchronize(cs(s)));
    })
}
gx_status gx_generate_permutation(gx_column_view out, uint64_t seed, int64_t base, gx_stream_t s) {
    GX_TRY({
        gx::generate_permutation(out, seed, base, cs(s));
        GX_CUDA(cudaStreamSynchronize(cs(s)));
    })
}
gx_status gx_generate_strings(const char* dict_chars, const int64_t* dict_offsets, int64_t dict_size,
                              const int32_t* codes, int64_t rows, const int64_t* out_offsets, char* out_chars,
                              gx_stream_t s) {
    GX_TRY({
        gx::generate_strings(dict_chars, dict_offsets, dict_size, codes, rows, out_offsets, out_chars, cs(s));
        GX_CUDA(cudaStreamSynchronize(cs(s)));
    })
}
gx_status gx_fill_sequence(gx_column_view out, int64_t start, int64_t step, gx_stream_t s) {
    GX_TRY({
        col c = resolve(out);
        gx::require(c.type == GX_INT64, "fill_sequence: INT64 column required");
        gx::sequence_i64(static_cast<int64_t*>(const_cast<void*>(c.data)), c.n, start, step, cs(s));
        GX_CUDA(cudaStreamSynchronize(cs(s)));
    })
}

}  // extern "C"
