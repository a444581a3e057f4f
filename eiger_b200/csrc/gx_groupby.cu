// gx_groupby.cu — the group-by dispatcher.
//
// Mirrors gamax::groupby::groupby / groupby_noskf
// (src/cuda/operators/groupby/groupby.cu:121-465): request rewriting (in
// gx_agg.cu), AUTO strategy selection, the allow_hash_fallback and
// PARTITION shape guards, SORT_OPT setting hint.optimize_sort, smart key
// fusion of multi-column keys, and the in/out hint contract.  STRING and
// multi-column keys group by a derived integer key (gx_keys.cu).  AUTO uses the reference's NDV threshold rule
// (groupby.cu:68-119) unless hint.selector asks for the learned selector.
#include <algorithm>

#include "gx_groupby.h"

namespace gx {

// Learned selector (gx_selector.cu): returns the variant (gx_groupby_algo)
// and writes the suggested radix bits.
int selector_choose(const col& key, const agg_plan& plan, int* radix_bits, cudaStream_t s);

static void auto_select(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req, int nreq,
                        gx_groupby_hint* hint, cudaStream_t s) {
    if (hint->groupby_algo != GX_GB_AUTO) return;
    for (int64_t i = 0; i < key->num_columns; ++i)
        if (key->columns[i].type == GX_STRING) { hint->groupby_algo = GX_GB_HASH; return; }
    if (key->num_columns != 1) { hint->groupby_algo = GX_GB_HASH; return; }
    col k = resolve(key->columns[0]);
    if (hint->selector == GX_SELECT_LEARNED) {
        int bits = 0;
        const agg_plan plan = make_agg_plan(val, req, nreq, hint->agg_count != 0);
        hint->groupby_algo = selector_choose(k, plan, &bits, s);
        if (hint->radix_bits <= 0) hint->radix_bits = bits;
        return;
    }
    int64_t est = ndv_estimate(k, s);
    bool four = size_of(k.type) == 4;
    int64_t thr = four ? (int64_t(1) << 14) : (int64_t(1) << 18);
    hint->groupby_algo = est <= thr ? GX_GB_HASH : GX_GB_PARTITION;
}

// One numeric key column through the chosen variant.
static void groupby_single(const col& k, const gx_table_view* val, const gx_agg_request* req, int nreq,
                           gx_groupby_hint* hint, cudaStream_t s, gx_table* out) {
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
}

// STRING or multi-column keys: group by one derived integer key (fused or
// chained dictionary codes) with ANY(row id) appended, then gather the
// original key columns at each group's row (groupby.cu:403-465 does the
// same with its fused key and ANY(tid)).  Output: [key columns..., one
// column per request..., COUNT when agg_count].
static void groupby_derived(const gx_table_view* key, owned_col&& dkey, int64_t bound, const gx_table_view* val,
                            const gx_agg_request* req, int nreq, gx_groupby_hint* hint, cudaStream_t s,
                            gx_table* out) {
    const int64_t n = key->columns[0].size;
    owned_col rid = make_col(GX_INT64, n, s);
    sequence_i64(rid.buf.get<int64_t>(), n, 0, 1, s);
    std::vector<gx_column_view> vcols;
    if (val)
        for (int64_t c = 0; c < val->num_columns; ++c) vcols.push_back(val->columns[c]);
    vcols.push_back(gx_column_view{rid.buf.get(), n, GX_INT64, 0});
    gx_table_view vt{vcols.data(), (int64_t)vcols.size()};
    std::vector<gx_agg_request> r(req, req + nreq);
    r.push_back(gx_agg_request{(int64_t)vcols.size() - 1, GX_AGG_ANY});
    gx_groupby_hint h = *hint;
    h.groups_upper_bound = std::min<int64_t>(hint->groups_upper_bound > 0 ? hint->groups_upper_bound : n, bound);
    gx_table tmp;
    col k{dkey.buf.get(), n, dkey.type};
    groupby_single(k, &vt, r.data(), (int)r.size(), &h, s, &tmp);
    hint->groupby_algo = h.groupby_algo;
    hint->optimize_sort = h.optimize_sort;
    hint->radix_bits = h.radix_bits;
    // tmp: [derived key, requests..., ANY(row id), (count)]
    const size_t any_idx = 1 + (size_t)nreq;
    const int64_t groups = tmp.cols[0].size;
    const int64_t* rows = tmp.cols[any_idx].buf.get<int64_t>();
    out->cols.clear();
    for (int64_t c = 0; c < key->num_columns; ++c)
        out->cols.push_back(gather_column(key->columns[c], rows, groups, s));
    for (size_t c = 1; c < tmp.cols.size(); ++c)
        if (c != any_idx) out->cols.push_back(std::move(tmp.cols[c]));
    GX_CUDA(cudaStreamSynchronize(s));
}

void groupby_dispatch(const gx_table_view* key, const gx_table_view* val, const gx_agg_request* req, int nreq,
                      gx_groupby_hint* hint, int forced_algo, cudaStream_t s, gx_table* out) {
    require(key && hint && out, "groupby: null argument");
    require(key->num_columns >= 1, "groupby: key table has no columns");
    const int64_t n = key->columns[0].size;
    for (int64_t c = 1; c < key->num_columns; ++c)
        require(key->columns[c].size == n, "groupby: key column " + std::to_string(c) +
                                               " has a different row count than key column 0");
    if (val)
        for (int64_t c = 0; c < val->num_columns; ++c)
            require(val->columns[c].size == n, "groupby: value column " + std::to_string(c) +
                                                   " has a different row count than the key");

    if (forced_algo >= 0) hint->groupby_algo = forced_algo;
    auto_select(key, val, req, nreq, hint, s);
    bool str = false;
    for (int64_t i = 0; i < key->num_columns; ++i) str |= key->columns[i].type == GX_STRING;
    const bool composite = str || key->num_columns > 1;
    if (hint->allow_hash_fallback && hint->groupby_algo != GX_GB_HASH && composite) hint->groupby_algo = GX_GB_HASH;
    if (!composite) {
        groupby_single(resolve(key->columns[0]), val, req, nreq, hint, s, out);
        GX_CUDA(cudaStreamSynchronize(s));
        return;
    }
    // Smart key fusion: integral key columns packed into one 64-bit key; any
    // variant may then run on it (groupby.cu:403-465).
    if (hint->enable_skf) {
        owned_col fused;
        int bits = 0;
        if (multikey_compress(key, 64, s, &fused, &bits)) {
            const int64_t bound = bits >= 62 ? n : std::min<int64_t>(n, int64_t(1) << bits);
            groupby_derived(key, std::move(fused), bound, val, req, nreq, hint, s, out);
            return;
        }
    }
    if (hint->groupby_algo == GX_GB_PARTITION || hint->groupby_algo == GX_GB_PARTITION_GFUR) {
        if (key->num_columns != 1)
            fail(GX_EINVAL, "PARTITION groupby: only single-column keys supported (got " +
                                std::to_string(key->num_columns) + ")");
        fail(GX_EINVAL, "PARTITION groupby: STRING keys not supported");
    }
    int64_t bound = n;
    owned_col dk = derive_group_key(key, false, s, &bound);
    groupby_derived(key, std::move(dk), bound, val, req, nreq, hint, s, out);
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
