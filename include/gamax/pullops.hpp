// pullops.hpp — volcano-style (pull) wrappers of the operators: each
// operator has open() / next() / close(); next() returns the next batch as
// an owned table, or nullptr when the input is exhausted.  The reference
// lists such a layer ("pullops - volcano-style wrappers of the operators",
// README.md:33) without shipping it; these wrappers sit on gamax.hpp and
// phys.hpp, so every batch runs through this library's kernels.
//
//   Scan       batches of an existing table (device copies of row slices)
//   Filter     phys::filter on every batch of its child
//   Project    picks and reorders columns of every batch
//   Aggregate  blocking: drains its child, then one phys::group_by
//   HashJoin   drains its build child on open(), joins each probe batch
//   Distinct   blocking: drains its child, then one phys::distinct
//
// Blocking operators concatenate numeric batches on the device (STRING
// batches are rejected there with std::runtime_error).
#pragma once

#include <algorithm>

#include "phys.hpp"

namespace gamax::pullops {

using table_ptr = std::unique_ptr<gamax::table>;

class Operator {
public:
    virtual ~Operator() = default;
    virtual void open() = 0;
    virtual table_ptr next() = 0;  // nullptr: no more batches
    virtual void close() {}
};
using op_ptr = std::unique_ptr<Operator>;

namespace detail {
// Device copy of rows [begin, begin + rows) of a numeric or STRING column.
inline column_ptr slice(column_view c, size_type begin, size_type rows, cudaStream_t s) {
    auto map = std::make_unique<column>(data_type{type_id::INT64}, rows, false, s);
    gamax::detail::check(gx_fill_sequence(map->view().to_gx(), begin, 1, gamax::detail::gs(s)));
    return util::device::gather(map->view(), c, s);
}

// All batches stacked into one table (numeric columns).
inline table_ptr concat(std::vector<table_ptr>& parts, cudaStream_t s) {
    if (parts.empty()) return nullptr;
    const size_type nc = parts[0]->num_columns();
    size_type rows = 0;
    for (auto& p : parts) rows += p->num_rows();
    std::vector<column_ptr> cols;
    for (size_type c = 0; c < nc; ++c) {
        const data_type t = parts[0]->get_column(c).type();
        if (t.id() == type_id::STRING) throw std::runtime_error("pullops: STRING columns cannot be concatenated");
        auto out = std::make_unique<column>(t, rows, false, s);
        size_type at = 0;
        const size_type w = size_of(t);
        for (auto& p : parts) {
            const size_type n = p->num_rows();
            if (n) cudaMemcpyAsync(static_cast<char*>(out->data()) + at * w, p->get_column(c).data(), (size_t)(n * w),
                                   cudaMemcpyDeviceToDevice, s);
            at += n;
        }
        cols.push_back(std::move(out));
    }
    cudaStreamSynchronize(s);
    return std::make_unique<table>(std::move(cols));
}

inline table_ptr drain(Operator& op, cudaStream_t s) {
    std::vector<table_ptr> parts;
    while (auto t = op.next()) parts.push_back(std::move(t));
    return concat(parts, s);
}
}  // namespace detail

class Scan : public Operator {
public:
    Scan(table_view src, size_type batch_rows, phys::Context ctx = {})
        : _src(src), _batch(batch_rows > 0 ? batch_rows : 1), _ctx(ctx) {}
    void open() override { _pos = 0; }
    table_ptr next() override {
        if (_pos >= _src.num_rows()) return nullptr;
        const size_type rows = std::min(_batch, _src.num_rows() - _pos);
        std::vector<column_ptr> cols;
        for (size_type c = 0; c < _src.num_columns(); ++c)
            cols.push_back(detail::slice(_src.get_column(c), _pos, rows, _ctx.stream));
        _pos += rows;
        return std::make_unique<table>(std::move(cols));
    }

private:
    table_view _src;
    size_type _batch, _pos{0};
    phys::Context _ctx;
};

class Filter : public Operator {
public:
    Filter(op_ptr child, std::vector<select::predicate> preds, select::combine how = select::combine::AND,
           phys::Context ctx = {})
        : _child(std::move(child)), _preds(std::move(preds)), _how(how), _ctx(ctx) {}
    void open() override { _child->open(); }
    table_ptr next() override {
        while (auto t = _child->next()) {
            auto out = phys::filter(t->view(), _preds, {}, _ctx, _how);
            if (out->num_rows() > 0) return out;
        }
        return nullptr;
    }
    void close() override { _child->close(); }

private:
    op_ptr _child;
    std::vector<select::predicate> _preds;
    select::combine _how;
    phys::Context _ctx;
};

class Project : public Operator {
public:
    Project(op_ptr child, std::vector<size_type> ordinals) : _child(std::move(child)), _ord(std::move(ordinals)) {}
    void open() override { _child->open(); }
    table_ptr next() override {
        auto t = _child->next();
        if (!t) return nullptr;
        std::vector<column_ptr> cols;
        std::vector<bool> taken((size_t)t->num_columns(), false);
        for (auto o : _ord) {
            if (o < 0 || o >= t->num_columns()) throw std::runtime_error("pullops::Project: ordinal out of range");
            if (taken[(size_t)o]) throw std::runtime_error("pullops::Project: a column is picked twice");
            taken[(size_t)o] = true;
            cols.push_back(t->release_column(o));
        }
        return std::make_unique<table>(std::move(cols));
    }
    void close() override { _child->close(); }

private:
    op_ptr _child;
    std::vector<size_type> _ord;
};

// Group-by over the child's rows: key and value column ordinals of the
// child's batches, aggregate specs over the value columns.
class Aggregate : public Operator {
public:
    Aggregate(op_ptr child, std::vector<size_type> keys, std::vector<size_type> values,
              std::vector<phys::AggSpec> specs, groupby::groupby_hint hint = {}, phys::Context ctx = {})
        : _child(std::move(child)), _keys(std::move(keys)), _vals(std::move(values)), _specs(std::move(specs)),
          _hint(hint), _ctx(ctx) {}
    void open() override {
        _child->open();
        _done = false;
    }
    table_ptr next() override {
        if (_done) return nullptr;
        _done = true;
        auto all = detail::drain(*_child, _ctx.stream);
        if (!all) return nullptr;
        auto v = all->view();
        return phys::group_by(v.select_columns(_keys), v.select_columns(_vals), _specs, _ctx, _hint);
    }
    void close() override { _child->close(); }

private:
    op_ptr _child;
    std::vector<size_type> _keys, _vals;
    std::vector<phys::AggSpec> _specs;
    groupby::groupby_hint _hint;
    phys::Context _ctx;
    bool _done{false};
};

class Distinct : public Operator {
public:
    Distinct(op_ptr child, groupby::groupby_hint hint = {}, phys::Context ctx = {})
        : _child(std::move(child)), _hint(hint), _ctx(ctx) {}
    void open() override {
        _child->open();
        _done = false;
    }
    table_ptr next() override {
        if (_done) return nullptr;
        _done = true;
        auto all = detail::drain(*_child, _ctx.stream);
        return all ? phys::distinct(all->view(), _ctx, _hint) : nullptr;
    }
    void close() override { _child->close(); }

private:
    op_ptr _child;
    groupby::groupby_hint _hint;
    phys::Context _ctx;
    bool _done{false};
};

// Inner equi-join: the build child is drained on open(); every probe batch
// is joined with it (phys::eq_join: [key, build non-keys..., probe non-keys...]).
class HashJoin : public Operator {
public:
    HashJoin(op_ptr build, size_type build_key, op_ptr probe, size_type probe_key,
             join::join_hint hint = phys::default_eq_join_hint(), phys::Context ctx = {})
        : _build(std::move(build)), _probe(std::move(probe)), _bkey(build_key), _pkey(probe_key), _hint(hint),
          _ctx(ctx) {}
    void open() override {
        _build->open();
        _table = detail::drain(*_build, _ctx.stream);
        _build->close();
        _probe->open();
    }
    table_ptr next() override {
        if (!_table) return nullptr;
        while (auto p = _probe->next()) {
            auto out = phys::eq_join(_table->view(), {_bkey}, p->view(), {_pkey}, _ctx, _hint);
            if (out->num_rows() > 0) return out;
        }
        return nullptr;
    }
    void close() override {
        _probe->close();
        _table.reset();
    }

private:
    op_ptr _build, _probe;
    size_type _bkey, _pkey;
    join::join_hint _hint;
    phys::Context _ctx;
    table_ptr _table;
};

}  // namespace gamax::pullops
