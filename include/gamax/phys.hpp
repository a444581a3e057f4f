// phys.hpp — the reference's physical-operator callers (namespace
// gamax::phys, src/cuda/phys/phys.hpp:47-260, phys.cu:29-663) for the
// operators this library implements: group_by, distinct, eq_join and
// filter, with the same empty-input short cuts, key reordering, payload
// sentinels, hint defaults and error messages, on top of gamax.hpp.
#pragma once

#include <algorithm>

#include "gamax.hpp"

namespace gamax::phys {

struct Context {
    cudaStream_t stream{0};
};

using table_ptr = std::unique_ptr<gamax::table>;

struct AggSpec {
    gamax::size_type column;
    gamax::groupby::aggregation_id agg;
};

// inner_eq_join rejects AUTO, so the engine default is a concrete pair
// (phys.hpp:82-87).
inline gamax::join::join_hint default_eq_join_hint() {
    gamax::join::join_hint h;
    h.join_algo = gamax::join::HASH;
    h.mat_algo = gamax::join::GFTR;
    return h;
}

namespace detail {
[[noreturn]] inline void phys_error(const std::string& what) { throw std::runtime_error("phys::" + what); }
[[noreturn]] inline void not_implemented(const std::string& op, const std::string& why) {
    throw std::runtime_error("phys::" + op + ": not yet implemented — " + why);
}

// A 0-row column of `type` (a STRING column holds its single 0 offset).
inline column_ptr zero_row_column(data_type type, cudaStream_t stream) {
    if (type.id() == type_id::STRING) {
        void* p = nullptr;
        gamax::detail::check(gx_malloc(&p, 8, gamax::detail::gs(stream)));
        cudaMemsetAsync(p, 0, 8, stream);
        return std::make_unique<column>(type, 0, p, 8);
    }
    return std::make_unique<column>(type, 0, false, stream);
}

inline column_ptr sequence(size_type n, cudaStream_t stream) {
    auto c = std::make_unique<column>(data_type{type_id::INT64}, n, false, stream);
    gamax::detail::check(gx_fill_sequence(c->view().to_gx(), 0, 1, gamax::detail::gs(stream)));
    return c;
}

inline void require_single_key(const std::string& op, const std::vector<size_type>& lkeys,
                               const std::vector<size_type>& rkeys) {
    if (lkeys.size() != rkeys.size())
        phys_error(op + ": lkeys (" + std::to_string(lkeys.size()) + ") and rkeys (" + std::to_string(rkeys.size()) +
                   ") must have the same length");
    if (lkeys.size() != 1)
        not_implemented(op, "multi-column keys (underlying inner_eq_join is single-key)");
}

inline std::vector<size_type> reorder_key_first(table_view in, size_type key) {
    std::vector<size_type> idx{key};
    for (size_type i = 0; i < in.num_columns(); ++i)
        if (i != key) idx.push_back(i);
    return idx;
}
}  // namespace detail

// Grouped aggregate (phys.cu:585-620): 0 input rows give a 0-row table of
// the output schema; otherwise groupby::groupby with a copy of the hint.
inline table_ptr group_by(table_view keys, table_view values, std::vector<AggSpec> specs, const Context& ctx,
                          const groupby::groupby_hint& hint_in = {}) {
    if (keys.num_rows() == 0) {
        std::vector<column_ptr> cols;
        for (size_type i = 0; i < keys.num_columns(); ++i)
            cols.push_back(detail::zero_row_column(keys.get_column(i).type(), ctx.stream));
        for (const auto& s : specs) {
            if (s.agg == groupby::aggregation_id::COUNT_ALL) {
                cols.push_back(detail::zero_row_column(data_type{type_id::INT64}, ctx.stream));
                continue;
            }
            auto out = groupby::agg_output_data_type(s.agg, values.get_column(s.column).type());
            cols.push_back(detail::zero_row_column(out, ctx.stream));
        }
        return std::make_unique<table>(std::move(cols));
    }
    std::vector<groupby::aggregation_request> requests;
    for (const auto& s : specs) requests.emplace_back(s.column, s.agg);
    auto hint = hint_in;
    return groupby::groupby(keys, values, requests, hint, ctx.stream);
}

// Distinct key rows (phys.cu:622-663): HASH / AUTO -> hash::distinct, the
// SORT family -> sort::distinct, PARTITION rejected.
inline table_ptr distinct(table_view keys, const Context& ctx, const groupby::groupby_hint& hint_in = {}) {
    if (keys.num_rows() == 0) {
        std::vector<column_ptr> cols;
        for (size_type i = 0; i < keys.num_columns(); ++i)
            cols.push_back(detail::zero_row_column(keys.get_column(i).type(), ctx.stream));
        return std::make_unique<table>(std::move(cols));
    }
    auto hint = hint_in;
    switch (hint.groupby_algo) {
        case groupby::HASH:
        case groupby::AUTO_ALGO: return groupby::hash::distinct(keys, hint, ctx.stream);
        case groupby::SORT:
        case groupby::SORT_OPT:
        case groupby::SORT_GFUR: return groupby::sort::distinct(keys, hint, ctx.stream);
        case groupby::PARTITION:
        case groupby::PARTITION_GFUR:
            throw std::runtime_error("phys::distinct: PARTITION variants are not supported; use HASH or SORT");
        default: throw std::runtime_error("phys::distinct: unknown groupby_algo");
    }
}

// Inner equi-join on one key column per side (phys.cu:422-470).  Output:
// [shared key, L non-key columns..., R non-key columns...].  A side with
// only its key gets a row-id payload for the join, removed afterwards.
inline table_ptr eq_join(table_view L, std::vector<size_type> lkeys, table_view R, std::vector<size_type> rkeys,
                         const Context& ctx, const join::join_hint& hint = default_eq_join_hint()) {
    detail::require_single_key("eq_join", lkeys, rkeys);
    if (L.num_rows() == 0 || R.num_rows() == 0) {
        std::vector<column_ptr> cols;
        cols.push_back(detail::zero_row_column(L.get_column(lkeys[0]).type(), ctx.stream));
        for (size_type i = 0; i < L.num_columns(); ++i)
            if (i != lkeys[0]) cols.push_back(detail::zero_row_column(L.get_column(i).type(), ctx.stream));
        for (size_type i = 0; i < R.num_columns(); ++i)
            if (i != rkeys[0]) cols.push_back(detail::zero_row_column(R.get_column(i).type(), ctx.stream));
        return std::make_unique<table>(std::move(cols));
    }
    auto lv = L.select_columns(detail::reorder_key_first(L, lkeys[0]));
    auto rv = R.select_columns(detail::reorder_key_first(R, rkeys[0]));
    column_ptr ls, rs;
    if (lv.num_columns() == 1) {
        ls = detail::sequence(L.num_rows(), ctx.stream);
        lv.add_column(ls->view());
    }
    if (rv.num_columns() == 1) {
        rs = detail::sequence(R.num_rows(), ctx.stream);
        rv.add_column(rs->view());
    }
    auto out = join::inner_eq_join(lv, rv, hint, ctx.stream);
    if (rs) out->remove_column(out->num_columns() - 1);
    if (ls) out->remove_column(1);
    return out;
}

// Rows of `in` the predicates keep (phys.cu:300-340); `output_ordinals`
// picks the columns materialised (empty = all), while the predicates may
// read any column.
inline table_ptr filter(table_view in, std::vector<select::predicate> const& preds,
                        std::vector<size_type> output_ordinals, const Context& ctx,
                        select::combine how = select::combine::AND) {
    for (auto o : output_ordinals)
        if (o < 0 || o >= in.num_columns())
            detail::phys_error("filter: output ordinal " + std::to_string(o) + " out of range for " +
                               std::to_string(in.num_columns()) + "-column input");
    std::vector<size_type> ords = output_ordinals;
    if (ords.empty())
        for (size_type i = 0; i < in.num_columns(); ++i) ords.push_back(i);
    if (in.num_rows() == 0) {
        std::vector<column_ptr> cols;
        for (auto o : ords) cols.push_back(detail::zero_row_column(in.get_column(o).type(), ctx.stream));
        return std::make_unique<table>(std::move(cols));
    }
    if (output_ordinals.empty()) return select::select(in, preds, how, ctx.stream);
    auto mask = select::select_to_bitmask(in, preds, how, ctx.stream);
    return util::device::compact(in.select_columns(ords), mask->view(), ctx.stream);
}

}  // namespace gamax::phys
