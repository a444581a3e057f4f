// gx_groupby.cu — the group-by dispatcher.
//
// Mirrors gamax::groupby::groupby / groupby_noskf
// (src/cuda/operators/groupby/groupby.cu:121-465): request rewriting (in
// gx_agg.cu), AUTO strategy selection, the allow_hash_fallback and
// PARTITION shape guards, SORT_OPT setting hint.optimize_sort, and the
// in/out hint contract.  AUTO uses the reference's NDV threshold rule
// (groupby.cu:68-119) unless hint.selector asks for the learned selector.
#include <algorithm>

#include "gx_groupby.h"

namespace gx {

// Learned selector (gx_selector.cu): returns the variant (gx_groupby_algo)
// and writes the suggested radix bits.
int selector_choose(const col& key, int* radix_bits, cudaStream_t s);

static void auto_select(const gx_table_view* key, gx_groupby_hint* hint, cudaStream_t s) {
    if (hint->groupby_algo != GX_GB_AUTO) return;
    for (int64_t i = 0; i < key->num_columns; ++i)
        if (key->columns[i].type == GX_STRING) { hint->groupby_algo = GX_GB_HASH; return; }
    if (key->num_columns != 1) { hint->groupby_algo = GX_GB_HASH; return; }
    col k = resolve(key->columns[0]);
    if (hint->selector == GX_SELECT_LEARNED) {
        int bits = 0;
        hint->groupby_algo = selector_choose(k, &bits, s);
        if (hint->radix_bits <= 0) hint->radix_bits = bits;
        return;
    }
    int64_t est = ndv_estimate(k, s);
    bool four = size_of(k.type) == 4;
    int64_t thr = four ? (int64_t(1) << 14) : (int64_t(1) << 18);
    hint->groupby_algo = est <= thr ? GX_GB_HASH : GX_GB_PARTITION;
}

void groupby_dispatch(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req, int nreq,
                      gx_groupby_hint* hint, int forced_algo, cudaStream_t s, gx_table* out) {
    require(key && hint && out, "groupby: null argument");
    require(key->num_columns >= 1, "groupby: key table has no columns");
    const int64_t n = key->columns[0].size;
    if (val)
        for (int64_t c = 0; c < val->num_columns; ++c)
            require(val->columns[c].size == n, "groupby: value column " + std::to_string(c) +
                                                   " has a different row count than the key");
    if (hint->enable_skf && key->num_columns > 1)
        fail(GX_EUNSUPPORTED, "multi-column keys (smart key fusion) are outside this library's scope");

    if (forced_algo >= 0) hint->groupby_algo = forced_algo;
    auto_select(key, hint, s);
    if (hint->allow_hash_fallback && hint->groupby_algo != GX_GB_HASH) {
        bool str = false;
        for (int64_t i = 0; i < key->num_columns; ++i) str |= key->columns[i].type == GX_STRING;
        if (str || key->num_columns > 1) hint->groupby_algo = GX_GB_HASH;
    }
    if (hint->groupby_algo == GX_GB_PARTITION || hint->groupby_algo == GX_GB_PARTITION_GFUR) {
        if (key->num_columns != 1)
            fail(GX_EINVAL, "PARTITION groupby: only single-column keys supported (got " +
                                std::to_string(key->num_columns) + ")");
        if (key->columns[0].type == GX_STRING) fail(GX_EINVAL, "PARTITION groupby: STRING keys not supported");
    }
    if (key->num_columns != 1)
        fail(GX_EUNSUPPORTED, "multi-column keys are outside this library's scope");
    if (key->columns[0].type == GX_STRING)
        fail(GX_EUNSUPPORTED, "STRING group keys are outside this library's scope (use gx_batch_* for string pipelines)");
    col k = resolve(key->columns[0]);
    require(is_numeric(k.type), "groupby: unsupported key type " + type_name(k.type));

    agg_plan p = make_agg_plan(val, req, nreq, hint->agg_count != 0);
    switch (hint->groupby_algo) {
        case GX_GB_SORT_OPT:
            hint->optimize_sort = 1;
            sort_groupby(k, p, hint, false, s, out);
            break;
        case GX_GB_SORT: sort_groupby(k, p, hint, false, s, out); break;
        case GX_GB_SORT_GFUR: sort_groupby(k, p, hint, true, s, out); break;
        case GX_GB_PARTITION: partition_groupby(k, p, hint, false, s, out); break;
        case GX_GB_PARTITION_GFUR: partition_groupby(k, p, hint, true, s, out); break;
        case GX_GB_HASH: hash_groupby(k, p, hint, s, out); break;
        default: fail(GX_EINVAL, "Unsupported groupby algorithm");
    }
    GX_CUDA(cudaStreamSynchronize(s));
}

// Distinct keys: a group-by without aggregations.
void distinct_dispatch(const gx_table_view* key, gx_groupby_hint* hint, int algo, cudaStream_t s, gx_table* out) {
    gx_groupby_hint h = *hint;
    h.agg_count = 0;
    groupby_dispatch(key, nullptr, nullptr, 0, &h, algo, s, out);
    hint->groupby_algo = h.groupby_algo;
}

// Scalar aggregate over whole columns: one group (constant key).
void aggregate_dispatch(const gx_table_view* input, const gx_agg_request* req, int nreq, cudaStream_t s,
                        gx_table* out) {
    require(input, "aggregate: null input");
    int64_t n = input->num_columns > 0 ? input->columns[0].size : 0;
    dbuf zeros((size_t)std::max<int64_t>(n, 1) * 4, s);
    GX_CUDA(cudaMemsetAsync(zeros.get(), 0, (size_t)std::max<int64_t>(n, 1) * 4, s));
    gx_column_view kv{zeros.get(), n, GX_INT32, 0};
    gx_table_view kt{&kv, 1};
    gx_groupby_hint h;
    gx_groupby_hint_init(&h);
    h.groups_upper_bound = 1;
    h.groupby_algo = GX_GB_HASH;
    gx_table tmp;
    groupby_dispatch(&kt, input, req, nreq, &h, GX_GB_HASH, s, &tmp);
    out->cols.clear();
    for (size_t c = 1; c < tmp.cols.size(); ++c) out->cols.push_back(std::move(tmp.cols[c]));
}

}  // namespace gx
