// gamax.hpp — the reference's C++ operator API (namespace gamax) rebuilt on
// the gx C ABI, so callers written against the reference's operators/ and
// compress/ headers compile unchanged against this library.
//
// Mirrors (paths inside the reference project):
//   types/data_type.hpp:8-58            size_type, type_id, data_type, sort_order
//   memory/column.hpp:13-240            column_view, mutable_column_view, column
//   memory/table.hpp:76-225             table_view, table
//   operators/groupby/groupby.hpp:16-49 groupby_algo, groupby_hint, groupby()
//   operators/groupby/aggregation.hpp   aggregation_id, aggregation_request
//   operators/groupby/groupby_{hash,sort,partition}.hpp   variant entry points
//   operators/join/join.hpp, inner_join.hpp               join_hint, inner_eq_join()
//   operators/sort/sort.hpp:14-75       sort_column_pair, sort_column, argsort
//   operators/partition/partition.hpp   partition_column_pair, ..., compute_partition_offsets
//   compress/dictionary_encode.hpp      dictionary_encode{,_with_order}, ready-dictionary and table overloads
//   compress/multikey_compress.hpp      multikey_compress (smart key fusion)
//   operators/groupby/aggregation.hpp   aggregate::aggregate; groupby_{hash,sort}.hpp distinct
//   utils/transform.hpp                 util::device::gather, compact, count_nonzero
//   operators/select/select.hpp         select / select_to_bitmask over predicate lists
// Error convention: a non-OK status throws std::bad_alloc for GX_ENOMEM and
// std::runtime_error otherwise (the reference's exception types).  Results
// are owned device columns freed through gx_free.
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>
#include <limits>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../gx.h"

namespace gamax {

using size_type = int64_t;
constexpr size_type MAXIMUM_SIZE = std::numeric_limits<size_type>::max();

enum class type_id {
    EMPTY, INT8, INT16, INT32, INT64, BOOL8, UINT8, UINT16, UINT32, UINT64, FLOAT32, FLOAT64, STRING, NUM_TYPE_IDS
};

class data_type {
public:
    data_type() = default;
    explicit constexpr data_type(type_id id) : _id{id} {}
    constexpr type_id id() const noexcept { return _id; }

private:
    type_id _id{type_id::EMPTY};
};
constexpr bool operator==(data_type const& a, data_type const& b) { return a.id() == b.id(); }
inline bool operator!=(data_type const& a, data_type const& b) { return !(a == b); }

enum class sort_order { ASCENDING, DESCENDING };

inline size_type size_of(data_type t) {
    switch (t.id()) {
        case type_id::INT8: case type_id::UINT8: case type_id::BOOL8: return 1;
        case type_id::INT16: case type_id::UINT16: return 2;
        case type_id::INT32: case type_id::UINT32: case type_id::FLOAT32: return 4;
        case type_id::INT64: case type_id::UINT64: case type_id::FLOAT64: return 8;
        default: return 0;
    }
}

namespace detail {
inline void check(gx_status s) {
    if (s == GX_OK) return;
    if (s == GX_ENOMEM) throw std::bad_alloc();
    throw std::runtime_error(gx_last_error_message());
}
inline gx_stream_t gs(cudaStream_t s) { return reinterpret_cast<gx_stream_t>(s); }
}  // namespace detail

class column_view_base {
public:
    column_view_base() = default;
    column_view_base(void* data, size_type size, data_type type, size_type offset = 0)
        : _data(data), _size(size - offset), _type(type), _offset(offset) {
        if (offset > size) throw std::runtime_error("Offset is greater than the size of the column");
    }
    size_type size() const noexcept { return _size; }
    data_type type() const noexcept { return _type; }
    gx_column_view to_gx() const { return gx_column_view{_data, _size, (int32_t)_type.id(), _offset}; }

protected:
    void* _data{nullptr};
    size_type _size{0};
    data_type _type;
    size_type _offset{0};
};

class column_view : public column_view_base {
public:
    using column_view_base::column_view_base;
    template <typename T>
    const T* data() const noexcept { return static_cast<const T*>(_data) + _offset; }
    const void* data() const noexcept { return static_cast<const char*>(_data) + _offset * size_of(_type); }
};

class mutable_column_view : public column_view_base {
public:
    using column_view_base::column_view_base;
    template <typename T>
    T* data() const noexcept { return static_cast<T*>(_data) + _offset; }
    void* data() const noexcept { return static_cast<char*>(_data) + _offset * size_of(_type); }
    void set_size(size_type size) noexcept { _size = size; }
    column_view view() const { return column_view(_data, _size + _offset, _type, _offset); }
};

// Owning device column (buffer from the library's stream-ordered pool).
class column {
public:
    // A STRING column's buffer holds its size+1 int64 offsets followed by the
    // characters (ARROW layout); its views point to a host-side
    // gx_string_columns pair, as the reference's string views point to a
    // (chars, offsets) helper (string/string_column.hpp:22-90).
    column(data_type type, size_type size, void* data, size_type capacity_bytes)
        : _type(type), _size(size), _data(data), _bytes(capacity_bytes) {
        if (type.id() == type_id::STRING)
            _str.reset(new gx_string_columns{static_cast<const char*>(data) + (size + 1) * 8,
                                             static_cast<const int64_t*>(data)});
    }
    explicit column(gx_column c) : column(data_type{(type_id)c.type}, c.size, c.data, c.capacity_bytes) {}
    column(data_type type, size_type num_rows, bool clear = false, cudaStream_t stream = 0)
        : _type(type), _size(num_rows) {
        _bytes = num_rows * size_of(type);
        if (_bytes) detail::check(gx_malloc(&_data, (size_t)_bytes, detail::gs(stream)));
        if (clear && _bytes) cudaMemsetAsync(_data, 0, (size_t)_bytes, stream);
    }
    column(const column&) = delete;
    column& operator=(const column&) = delete;
    column(column&& o) noexcept
        : _type(o._type), _size(o._size), _data(o._data), _bytes(o._bytes), _str(std::move(o._str)) {
        o._data = nullptr;
        o._size = 0;
    }
    virtual ~column() {
        if (_data) gx_free(_data, nullptr);
    }
    size_type size() const noexcept { return _size; }
    data_type type() const noexcept { return _type; }
    void set_size(size_type s) noexcept { _size = s; }
    size_type bytes() const noexcept { return _bytes; }
    template <typename T = void>
    T* data() const noexcept { return static_cast<T*>(_data); }
    column_view view(size_type offset = 0) const {
        return column_view(_str ? static_cast<void*>(_str.get()) : _data, _size, _type, offset);
    }
    mutable_column_view mutable_view(size_type offset = 0) {
        return mutable_column_view(_str ? static_cast<void*>(_str.get()) : _data, _size, _type, offset);
    }

private:
    data_type _type;
    size_type _size{0};
    void* _data{nullptr};
    size_type _bytes{0};
    std::unique_ptr<gx_string_columns> _str;
};
using column_ptr = std::unique_ptr<column>;

template <typename column_view_t>
class table_view_base {
public:
    table_view_base() = default;
    table_view_base(std::vector<column_view_t> const& cols) : _columns(cols) {}
    table_view_base(std::vector<std::unique_ptr<column>> const& cols) {
        for (auto& c : cols) {
            if constexpr (std::is_same<column_view_t, column_view>::value) _columns.push_back(c->view());
            else _columns.push_back(c->mutable_view());
        }
    }
    size_type num_columns() const noexcept { return (size_type)_columns.size(); }
    size_type num_rows() const noexcept { return _columns.empty() ? 0 : _columns[0].size(); }
    column_view_t get_column(size_type i) const { return _columns.at(i); }
    column_view_t operator[](size_type i) const { return get_column(i); }
    void add_column(column_view_t c) {
        if (c.size() != num_rows()) throw std::runtime_error("New column must have the same number of rows as the table");
        _columns.push_back(c);
    }
    table_view_base select_columns(std::vector<size_type> const& idx) const {
        std::vector<column_view_t> cols;
        for (auto i : idx) cols.push_back(_columns.at(i));
        return table_view_base(cols);
    }
    std::vector<gx_column_view> to_gx() const {
        std::vector<gx_column_view> v;
        for (auto& c : _columns) v.push_back(c.to_gx());
        return v;
    }

private:
    std::vector<column_view_t> _columns;
};
using table_view = table_view_base<column_view>;
using mutable_table_view = table_view_base<mutable_column_view>;

class table {
public:
    table() = default;
    table(std::vector<std::unique_ptr<column>>&& cols) : _columns(std::move(cols)) {}
    size_type num_columns() const noexcept { return (size_type)_columns.size(); }
    size_type num_rows() const noexcept { return _columns.empty() ? 0 : _columns[0]->size(); }
    column& get_column(size_type i) const { return *_columns.at(i); }
    void add_column(std::unique_ptr<column>&& c) { _columns.push_back(std::move(c)); }
    std::unique_ptr<column> release_column(size_type i) { return std::move(_columns.at(i)); }
    std::unique_ptr<column> remove_column(size_type i) {
        auto c = std::move(_columns.at(i));
        _columns.erase(_columns.begin() + i);
        return c;
    }
    table_view view() const { return table_view(_columns); }

private:
    std::vector<std::unique_ptr<column>> _columns;
};

namespace detail {
// Moves every column of a gx_table into a gamax::table.
inline std::unique_ptr<table> adopt(gx_table* t) {
    auto out = std::make_unique<table>();
    int64_t n = gx_table_num_columns(t);
    for (int64_t i = 0; i < n; ++i) {
        gx_column c;
        gx_status s = gx_table_release_column(t, i, &c);
        if (s != GX_OK) {
            gx_table_free(t);
            check(s);
        }
        out->add_column(std::make_unique<column>(c));
    }
    gx_table_free(t);
    return out;
}
struct gx_tv {
    std::vector<gx_column_view> cols;
    gx_table_view tv;
    explicit gx_tv(const table_view& t) : cols(t.to_gx()) { tv = gx_table_view{cols.data(), (int64_t)cols.size()}; }
};
}  // namespace detail

// ------------------------------------------------------------------ groupby
namespace groupby {
enum groupby_algo { AUTO_ALGO, HASH, SORT, SORT_OPT, SORT_GFUR, PARTITION, PARTITION_GFUR, UNSUPPORTED_GROUPBY_ALGO };

struct groupby_hint {
    size_type groups_upper_bound{MAXIMUM_SIZE};
    bool zero_based_ids{false};
    bool optimize_sort{false};
    ::gamax::groupby::groupby_algo groupby_algo{AUTO_ALGO};
    bool agg_count{false};
    bool enable_skf{false};
    bool allow_hash_fallback{false};
};

enum class aggregation_id { SUM, MAX, MIN, AVG, ANY, COUNT_ALL, NOT_SUPPORTED_AGGREGATION };

struct aggregation_request {
    size_type column_index;
    aggregation_id agg_kind;
    aggregation_request(size_type c, aggregation_id k) : column_index(c), agg_kind(k) {}
};

inline data_type agg_output_data_type(aggregation_id const& k, data_type const& t) {
    return data_type{(type_id)gx_agg_output_type((int32_t)k, (int32_t)t.id())};
}

namespace detail {
using fn_t = gx_status (*)(const gx_table_view*, const gx_table_view*, const gx_agg_request*, int32_t,
                           gx_groupby_hint*, gx_stream_t, gx_table**);
inline std::unique_ptr<table> run(fn_t fn, table_view key, table_view val, std::vector<aggregation_request>& reqs,
                                  groupby_hint& hint, cudaStream_t stream) {
    gamax::detail::gx_tv k(key), v(val);
    std::vector<gx_agg_request> r;
    for (auto& q : reqs) r.push_back(gx_agg_request{q.column_index, (int32_t)q.agg_kind});
    gx_groupby_hint h;
    gx_groupby_hint_init(&h);
    h.groups_upper_bound = hint.groups_upper_bound;
    h.zero_based_ids = hint.zero_based_ids;
    h.optimize_sort = hint.optimize_sort;
    h.groupby_algo = (int32_t)hint.groupby_algo;
    h.agg_count = hint.agg_count;
    h.enable_skf = hint.enable_skf;
    h.allow_hash_fallback = hint.allow_hash_fallback;
    gx_table* out = nullptr;
    gamax::detail::check(fn(&k.tv, &v.tv, r.data(), (int32_t)r.size(), &h, gamax::detail::gs(stream), &out));
    // The hint is in/out like the reference's non-const reference.
    hint.groupby_algo = (groupby_algo)h.groupby_algo;
    hint.optimize_sort = h.optimize_sort != 0;
    hint.groups_upper_bound = h.groups_upper_bound;
    return gamax::detail::adopt(out);
}
}  // namespace detail

inline std::unique_ptr<table> groupby(table_view key, table_view val, std::vector<aggregation_request>& reqs,
                                      groupby_hint& hint, cudaStream_t stream = 0) {
    return detail::run(gx_groupby, key, val, reqs, hint, stream);
}
namespace detail {
using distinct_fn_t = gx_status (*)(const gx_table_view*, gx_groupby_hint*, gx_stream_t, gx_table**);
inline std::unique_ptr<table> run_distinct(distinct_fn_t fn, table_view key, groupby_hint& hint, cudaStream_t stream) {
    gamax::detail::gx_tv k(key);
    gx_groupby_hint h;
    gx_groupby_hint_init(&h);
    h.groups_upper_bound = hint.groups_upper_bound;
    h.groupby_algo = (int32_t)hint.groupby_algo;
    h.enable_skf = hint.enable_skf;
    gx_table* out = nullptr;
    gamax::detail::check(fn(&k.tv, &h, gamax::detail::gs(stream), &out));
    hint.groupby_algo = (groupby_algo)h.groupby_algo;
    return gamax::detail::adopt(out);
}
}  // namespace detail

namespace hash {
inline std::unique_ptr<table> groupby(table_view key, table_view val, std::vector<aggregation_request>& reqs,
                                      groupby_hint& hint, cudaStream_t stream = 0) {
    return detail::run(gx_groupby_hash, key, val, reqs, hint, stream);
}
// One row per distinct key row (groupby_hash.hpp:24-34); STRING and
// multi-column keys included.
inline std::unique_ptr<table> distinct(table_view key, groupby_hint& hint, cudaStream_t stream = 0) {
    return detail::run_distinct(gx_distinct_hash, key, hint, stream);
}
}  // namespace hash
namespace sort {
inline std::unique_ptr<table> groupby(table_view key, table_view val, std::vector<aggregation_request>& reqs,
                                      groupby_hint& hint, cudaStream_t stream = 0) {
    return detail::run(gx_groupby_sort, key, val, reqs, hint, stream);
}
inline std::unique_ptr<table> groupby_gfur(table_view key, table_view val, std::vector<aggregation_request>& reqs,
                                           groupby_hint& hint, cudaStream_t stream = 0) {
    return detail::run(gx_groupby_sort_gfur, key, val, reqs, hint, stream);
}
// Sort-based distinct (groupby_sort.hpp:31-47).
inline std::unique_ptr<table> distinct(table_view key, groupby_hint& hint, cudaStream_t stream = 0) {
    return detail::run_distinct(gx_distinct_sort, key, hint, stream);
}
}  // namespace sort
namespace partition {
inline std::unique_ptr<table> groupby(table_view key, table_view val, std::vector<aggregation_request>& reqs,
                                      groupby_hint& hint, cudaStream_t stream = 0) {
    return detail::run(gx_groupby_partition, key, val, reqs, hint, stream);
}
inline std::unique_ptr<table> groupby_gfur(table_view key, table_view val, std::vector<aggregation_request>& reqs,
                                           groupby_hint& hint, cudaStream_t stream = 0) {
    return detail::run(gx_groupby_partition_gfur, key, val, reqs, hint, stream);
}
}  // namespace partition

// Whole-table aggregates, one output row (aggregation.hpp:32-37).
namespace aggregate {
inline std::unique_ptr<table> aggregate(table_view input, std::vector<aggregation_request>& reqs,
                                        cudaStream_t stream = 0) {
    gamax::detail::gx_tv t(input);
    std::vector<gx_agg_request> r;
    for (auto& q : reqs) r.push_back(gx_agg_request{q.column_index, (int32_t)q.agg_kind});
    gx_table* out = nullptr;
    gamax::detail::check(gx_aggregate(&t.tv, r.data(), (int32_t)r.size(), gamax::detail::gs(stream), &out));
    return gamax::detail::adopt(out);
}
}  // namespace aggregate
}  // namespace groupby

// --------------------------------------------------------------------- join
namespace join {
constexpr size_type MAX_JOIN_OUTPUT_SIZE = (1 << 30);
enum join_algo { AUTO_ALGO, HASH, SORT, PARTITION, UNSUPPORTED_JOIN_ALGO };
enum materialization_algo { AUTO_MAT, GFUR, GFTR, INDEX_CLUSTER, UNSUPPORTED_MATERIALIZATION_ALGO };
struct join_hint {
    bool sorted_left{false};
    bool sorted_right{false};
    bool unique_left{false};
    bool unique_right{false};
    size_type max_out{0};
    ::gamax::join::join_algo join_algo{AUTO_ALGO};
    materialization_algo mat_algo{AUTO_MAT};
};
inline std::unique_ptr<table> inner_eq_join(table_view left, table_view right, join_hint const& hint,
                                            cudaStream_t stream = 0) {
    gamax::detail::gx_tv l(left), r(right);
    gx_join_hint h;
    gx_join_hint_init(&h);
    h.sorted_left = hint.sorted_left;
    h.sorted_right = hint.sorted_right;
    h.unique_left = hint.unique_left;
    h.unique_right = hint.unique_right;
    h.max_out = hint.max_out;
    h.join_algo = (int32_t)hint.join_algo;
    h.mat_algo = (int32_t)hint.mat_algo;
    gx_table* out = nullptr;
    gamax::detail::check(gx_inner_eq_join(&l.tv, &r.tv, &h, gamax::detail::gs(stream), &out));
    return gamax::detail::adopt(out);
}
}  // namespace join

// --------------------------------------------------------------------- sort
namespace sort {
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> sort_column_pair(
    column_view key, column_view val, int begin_bit = 0, int end_bit = -1,
    sort_order order = sort_order::ASCENDING, void* d_temp = nullptr, size_t temp_bytes = 0,
    cudaStream_t stream = 0) {
    gx_column k, v;
    gamax::detail::check(gx_sort_column_pair(key.to_gx(), val.to_gx(), begin_bit, end_bit, (int32_t)order, d_temp,
                                             temp_bytes, gamax::detail::gs(stream), &k, &v));
    return {std::make_unique<column>(k), std::make_unique<column>(v)};
}
inline std::unique_ptr<column> sort_column(column_view col, int begin_bit = 0, int end_bit = -1,
                                           sort_order order = sort_order::ASCENDING, void* d_temp = nullptr,
                                           size_t temp_bytes = 0, cudaStream_t stream = 0) {
    gx_column k;
    gamax::detail::check(gx_sort_column(col.to_gx(), begin_bit, end_bit, (int32_t)order, d_temp, temp_bytes,
                                        gamax::detail::gs(stream), &k));
    return std::make_unique<column>(k);
}
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> argsort(
    column_view col, int begin_bit = 0, int end_bit = -1, sort_order order = sort_order::ASCENDING,
    void* d_temp = nullptr, size_t temp_bytes = 0, cudaStream_t stream = 0) {
    gx_column k, i;
    gamax::detail::check(gx_argsort(col.to_gx(), begin_bit, end_bit, (int32_t)order, d_temp, temp_bytes,
                                    gamax::detail::gs(stream), &k, &i));
    return {std::make_unique<column>(k), std::make_unique<column>(i)};
}
// gamax::column& overloads (sort.hpp:14-75): the same sorts on the column's view.
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> sort_column_pair(
    column& key, column& val, int begin_bit = 0, int end_bit = -1, sort_order order = sort_order::ASCENDING,
    void* d_temp = nullptr, size_t temp_bytes = 0, cudaStream_t stream = 0) {
    return sort_column_pair(key.view(), val.view(), begin_bit, end_bit, order, d_temp, temp_bytes, stream);
}
inline std::unique_ptr<column> sort_column(column& col, int begin_bit = 0, int end_bit = -1,
                                           sort_order order = sort_order::ASCENDING, void* d_temp = nullptr,
                                           size_t temp_bytes = 0, cudaStream_t stream = 0) {
    return sort_column(col.view(), begin_bit, end_bit, order, d_temp, temp_bytes, stream);
}
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> argsort(
    column& col, int begin_bit = 0, int end_bit = -1, sort_order order = sort_order::ASCENDING,
    void* d_temp = nullptr, size_t temp_bytes = 0, cudaStream_t stream = 0) {
    return argsort(col.view(), begin_bit, end_bit, order, d_temp, temp_bytes, stream);
}
}  // namespace sort

// ---------------------------------------------------------------- partition
namespace partition {
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> partition_column_pair(
    column_view key, column_view val, int begin_bit, int end_bit, void* d_temp = nullptr, size_t temp_bytes = 0,
    cudaStream_t stream = 0) {
    gx_column k, v;
    gamax::detail::check(gx_partition_column_pair(key.to_gx(), val.to_gx(), begin_bit, end_bit, d_temp, temp_bytes,
                                                  gamax::detail::gs(stream), &k, &v));
    return {std::make_unique<column>(k), std::make_unique<column>(v)};
}
inline std::unique_ptr<column> partition_column(column_view col, int begin_bit, int end_bit, void* d_temp = nullptr,
                                                size_t temp_bytes = 0, cudaStream_t stream = 0) {
    gx_column k;
    gamax::detail::check(gx_partition_column(col.to_gx(), begin_bit, end_bit, d_temp, temp_bytes,
                                             gamax::detail::gs(stream), &k));
    return std::make_unique<column>(k);
}
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> arg_partition(
    column_view col, int begin_bit, int end_bit, void* d_temp = nullptr, size_t temp_bytes = 0,
    cudaStream_t stream = 0) {
    gx_column k, i;
    gamax::detail::check(gx_arg_partition(col.to_gx(), begin_bit, end_bit, d_temp, temp_bytes,
                                          gamax::detail::gs(stream), &k, &i));
    return {std::make_unique<column>(k), std::make_unique<column>(i)};
}
inline std::unique_ptr<column> compute_partition_offsets(column_view col, int begin_bit, int end_bit,
                                                         cudaStream_t stream = 0) {
    gx_column o;
    gamax::detail::check(gx_compute_partition_offsets(col.to_gx(), begin_bit, end_bit, gamax::detail::gs(stream), &o));
    return std::make_unique<column>(o);
}
// gamax::column& overloads (partition.hpp:11-45).
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> partition_column_pair(
    column& key, column& val, int begin_bit, int end_bit, void* d_temp = nullptr, size_t temp_bytes = 0,
    cudaStream_t stream = 0) {
    return partition_column_pair(key.view(), val.view(), begin_bit, end_bit, d_temp, temp_bytes, stream);
}
inline std::unique_ptr<column> partition_column(column& col, int begin_bit, int end_bit, void* d_temp = nullptr,
                                                size_t temp_bytes = 0, cudaStream_t stream = 0) {
    return partition_column(col.view(), begin_bit, end_bit, d_temp, temp_bytes, stream);
}
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> arg_partition(
    column& col, int begin_bit, int end_bit, void* d_temp = nullptr, size_t temp_bytes = 0, cudaStream_t stream = 0) {
    return arg_partition(col.view(), begin_bit, end_bit, d_temp, temp_bytes, stream);
}
inline std::unique_ptr<column> compute_partition_offsets(column& col, int begin_bit, int end_bit,
                                                         cudaStream_t stream = 0) {
    return compute_partition_offsets(col.view(), begin_bit, end_bit, stream);
}
}  // namespace partition

// ----------------------------------------------------------------- compress
namespace compress {
inline std::pair<std::unique_ptr<column>, size_type> dictionary_encode(
    const column_view col, const data_type encode_type = data_type{type_id::INT32},
    const size_type dictionary_size_hint = 0, const double load_factor = 0.25, cudaStream_t stream = 0) {
    gx_column c;
    int64_t nd = 0;
    gamax::detail::check(gx_dictionary_encode(col.to_gx(), (int32_t)encode_type.id(), dictionary_size_hint,
                                              load_factor, gamax::detail::gs(stream), &c, &nd));
    return {std::make_unique<column>(c), nd};
}
inline std::pair<std::unique_ptr<column>, size_type> dictionary_encode_with_order(
    const column_view col, const data_type encode_type = data_type{type_id::INT32},
    const size_type dictionary_size_hint = 0, const double load_factor = 0.25, cudaStream_t stream = 0) {
    gx_column c;
    int64_t nd = 0;
    gamax::detail::check(gx_dictionary_encode_with_order(col.to_gx(), (int32_t)encode_type.id(), dictionary_size_hint,
                                                         load_factor, gamax::detail::gs(stream), &c, &nd));
    return {std::make_unique<column>(c), nd};
}
inline std::unique_ptr<column> dictionary_encode(const column_view col, const column_view dict,
                                                 const data_type encode_type = data_type{type_id::INT32},
                                                 cudaStream_t stream = 0) {
    gx_column c;
    gamax::detail::check(gx_dictionary_encode_with_dict(col.to_gx(), dict.to_gx(), (int32_t)encode_type.id(),
                                                        gamax::detail::gs(stream), &c));
    return std::make_unique<column>(c);
}
// The table overload rejects every table, as the reference's does
// (dictionary_encode.cu:41-43, 376-384).
inline std::pair<std::unique_ptr<column>, size_type> dictionary_encode(
    const table_view, const data_type = data_type{type_id::INT32}, const size_type = 0, const double = 0.25,
    cudaStream_t = 0) {
    throw std::runtime_error("Cannot dictionary encode table");
}

struct multikey_compress_options {
    bool always_compress = true;
    int max_fused_key_bits = 64;
    int* out_total_bits = nullptr;
};
// Smart key fusion (multikey_compress.hpp:29-32): nullptr when the keys
// cannot be packed into max_fused_key_bits bits.
inline std::unique_ptr<column> multikey_compress(table_view table, multikey_compress_options const& options = {},
                                                 cudaStream_t stream = 0) {
    gamax::detail::gx_tv t(table);
    gx_column c;
    int32_t bits = 0;
    gx_status st = gx_multikey_compress(&t.tv, options.max_fused_key_bits, gamax::detail::gs(stream), &c, &bits);
    if (st == GX_EUNSUPPORTED) return nullptr;
    gamax::detail::check(st);
    if (options.out_total_bits) *options.out_total_bits = bits;
    return std::make_unique<column>(c);
}
}  // namespace compress

// ----------------------------------------------------------------- util
namespace util::device {
// out[i] = input[gather_map[i]] (utils/transform.hpp, transform.cu:168-186).
inline std::unique_ptr<column> gather(column_view gather_map, column_view input, cudaStream_t stream = 0) {
    gx_column c;
    gamax::detail::check(gx_gather(gather_map.to_gx(), input.to_gx(), gamax::detail::gs(stream), &c));
    return std::make_unique<column>(c);
}
// Rows of every column whose BOOL8 mask byte is nonzero, in order
// (transform.hpp:34-48).
inline std::unique_ptr<table> compact(table_view input, column_view mask, cudaStream_t stream = 0) {
    gamax::detail::gx_tv t(input);
    gx_table* out = nullptr;
    gamax::detail::check(gx_compact(&t.tv, mask.to_gx(), gamax::detail::gs(stream), &out));
    return gamax::detail::adopt(out);
}
inline std::unique_ptr<column> compact(column_view input, column_view mask, cudaStream_t stream = 0) {
    auto t = compact(table_view(std::vector<column_view>{input}), mask, stream);
    return t->release_column(0);
}
inline size_type count_nonzero(column_view input, cudaStream_t stream = 0) {
    int64_t c = 0;
    gamax::detail::check(gx_count_nonzero(input.to_gx(), gamax::detail::gs(stream), &c));
    return c;
}
}  // namespace util::device

// ------------------------------------------------------------------ select
// Filters whose predicate is a list of column-vs-literal comparisons joined
// by AND or OR (gx_predicate); the reference's select takes general
// expression trees (select.hpp:15-64), which this library does not build.
namespace select {
enum class cmp { LT, LE, GT, GE, EQ, NE, BETWEEN };
struct predicate {
    size_type column;
    cmp op;
    int64_t lo_i{0}, hi_i{0};
    double lo_f{0}, hi_f{0};
    static predicate on_int(size_type c, cmp op, int64_t lo, int64_t hi = 0) {
        return predicate{c, op, lo, hi, (double)lo, (double)hi};
    }
    static predicate on_float(size_type c, cmp op, double lo, double hi = 0) {
        return predicate{c, op, (int64_t)lo, (int64_t)hi, lo, hi};
    }
};
enum class combine { AND, OR };
namespace detail {
inline std::vector<gx_predicate> to_gx(std::vector<predicate> const& ps) {
    std::vector<gx_predicate> out;
    for (auto& p : ps) out.push_back(gx_predicate{p.column, (int32_t)p.op, 0, p.lo_i, p.hi_i, p.lo_f, p.hi_f});
    return out;
}
}  // namespace detail
inline column_ptr select_to_bitmask(table_view table, std::vector<predicate> const& preds,
                                    combine how = combine::AND, cudaStream_t stream = 0) {
    gamax::detail::gx_tv t(table);
    auto q = detail::to_gx(preds);
    gx_column c;
    gamax::detail::check(gx_select_to_bitmask(&t.tv, q.data(), (int32_t)q.size(), (int32_t)how,
                                              gamax::detail::gs(stream), &c));
    return std::make_unique<column>(c);
}
inline std::unique_ptr<table> select(table_view table, std::vector<predicate> const& preds,
                                     combine how = combine::AND, cudaStream_t stream = 0) {
    gamax::detail::gx_tv t(table);
    auto q = detail::to_gx(preds);
    gx_table* out = nullptr;
    gamax::detail::check(gx_select(&t.tv, q.data(), (int32_t)q.size(), (int32_t)how, gamax::detail::gs(stream), &out));
    return gamax::detail::adopt(out);
}
}  // namespace select

// -------------------------------------------------------------------- stats
namespace stats {
inline size_type compute_ndv_approx(column_view col, cudaStream_t stream = 0) {
    int64_t nd = 0;
    gamax::detail::check(gx_compute_ndv_approx(col.to_gx(), gamax::detail::gs(stream), &nd));
    return nd;
}
}  // namespace stats

}  // namespace gamax
