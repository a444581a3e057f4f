"""A reference-style C++ caller, compiled with g++ against
include/gamax/{gamax,phys,pullops}.hpp and libgx.so, runs the operators on
device data the way the reference's own callers do (gamax::groupby::groupby,
join::inner_eq_join, sort::sort_column_pair on gamax::column&, partition
offsets, compress::dictionary_encode_with_order, aggregate::aggregate,
hash::distinct, phys::{group_by, eq_join, filter, distinct} and a pullops
Scan -> Filter -> Aggregate pipeline).  Its outputs are checked here
against the CPU oracle on the same inputs."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
CUDA = Path("/usr/local/cuda")

CALLER = r'''
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "gamax/pullops.hpp"
using namespace gamax;

static std::string dir;
template <class T> std::vector<T> load(const char* name) {
    std::ifstream f(dir + "/" + name, std::ios::binary | std::ios::ate);
    size_t bytes = (size_t)f.tellg();
    std::vector<T> v(bytes / sizeof(T));
    f.seekg(0);
    f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)bytes);
    return v;
}
template <class T> T* upload(const std::vector<T>& h) {
    T* d = nullptr;
    cudaMalloc(&d, std::max<size_t>(h.size(), 1) * sizeof(T));
    cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}
static void save(const char* name, const void* dptr, size_t bytes) {
    std::vector<char> h(bytes);
    if (bytes) cudaMemcpy(h.data(), dptr, bytes, cudaMemcpyDeviceToHost);
    std::ofstream f(dir + "/" + name, std::ios::binary);
    f.write(h.data(), (std::streamsize)bytes);
}
static void save_col(const char* name, const column& c) { save(name, c.data(), (size_t)(c.size() * size_of(c.type()))); }
static data_type I32{type_id::INT32}, I64{type_id::INT64};
using agg = groupby::aggregation_id;

int main(int argc, char** argv) {
    dir = argv[1];
    auto key = load<int32_t>("key.bin");
    auto key2 = load<int32_t>("key2.bin");
    auto val = load<int64_t>("val.bin");
    auto pk = load<int32_t>("pk.bin");
    auto fk = load<int32_t>("fk.bin");
    const size_type n = (size_type)key.size();
    column_view kc(upload(key), n, I32), k2c(upload(key2), n, I32), vc(upload(val), n, I64);

    // group-by, hash and partition variants: SUM + COUNT
    for (auto algo : {groupby::HASH, groupby::PARTITION}) {
        std::vector<groupby::aggregation_request> reqs{{0, agg::SUM}, {0, agg::COUNT_ALL}};
        groupby::groupby_hint hint;
        hint.groupby_algo = algo;
        auto g = groupby::groupby(table_view({kc}), table_view({vc}), reqs, hint);
        std::string p = algo == groupby::HASH ? "gb_hash_" : "gb_part_";
        save_col((p + "key").c_str(), g->get_column(0));
        save_col((p + "sum").c_str(), g->get_column(1));
        save_col((p + "cnt").c_str(), g->get_column(2));
        if (hint.groupby_algo != algo) return 2;
    }
    // inner_eq_join [key, build payload, probe payload]
    {
        std::vector<int64_t> lrow(pk.size()), rrow(fk.size());
        for (size_t i = 0; i < lrow.size(); ++i) lrow[i] = (int64_t)i;
        for (size_t i = 0; i < rrow.size(); ++i) rrow[i] = (int64_t)i;
        column_view l0(upload(pk), (size_type)pk.size(), I32), l1(upload(lrow), (size_type)pk.size(), I64);
        column_view r0(upload(fk), (size_type)fk.size(), I32), r1(upload(rrow), (size_type)fk.size(), I64);
        join::join_hint h;
        h.join_algo = join::SORT;
        h.mat_algo = join::GFTR;
        auto j = join::inner_eq_join(table_view({l0, l1}), table_view({r0, r1}), h);
        save_col("join_l", j->get_column(1));
        save_col("join_r", j->get_column(2));
    }
    // sort::sort_column_pair on owned gamax::column& (sort.hpp:14-23)
    {
        column keys(I32, n), vals(I64, n);
        cudaMemcpy(keys.data(), kc.data(), n * 4, cudaMemcpyDeviceToDevice);
        cudaMemcpy(vals.data(), vc.data(), n * 8, cudaMemcpyDeviceToDevice);
        auto [sk, sv] = sort::sort_column_pair(keys, vals);
        save_col("sort_k", *sk);
        save_col("sort_v", *sv);
        auto off = partition::compute_partition_offsets(*sk, 0, 6);
        save_col("part_off", *off);
    }
    // order-preserving dictionary codes
    {
        auto [codes, ndv] = compress::dictionary_encode_with_order(kc, I32);
        save_col("dict_codes", *codes);
        std::printf("ndv %lld\n", (long long)ndv);
        try {
            compress::dictionary_encode(table_view({kc}));
            return 3;
        } catch (std::runtime_error const& e) {
            std::printf("table_encode:%s\n", e.what());
        }
    }
    // aggregate::aggregate SUM / MIN / MAX over the whole value column
    {
        std::vector<groupby::aggregation_request> reqs{{0, agg::SUM}, {0, agg::MIN}, {0, agg::MAX}};
        auto a = groupby::aggregate::aggregate(table_view({vc}), reqs);
        save_col("agg_sum", a->get_column(0));
        save_col("agg_min", a->get_column(1));
        save_col("agg_max", a->get_column(2));
    }
    // phys: two-column key with smart key fusion, distinct, join, filter
    phys::Context ctx;
    {
        groupby::groupby_hint h;
        h.enable_skf = true;
        auto g = phys::group_by(table_view({kc, k2c}), table_view({vc}), {{0, agg::SUM}, {0, agg::COUNT_ALL}}, ctx, h);
        save_col("mk_k1", g->get_column(0));
        save_col("mk_k2", g->get_column(1));
        save_col("mk_sum", g->get_column(2));
        save_col("mk_cnt", g->get_column(3));
        auto d = phys::distinct(table_view({kc}), ctx);
        save_col("distinct", d->get_column(0));
        auto e = phys::group_by(table_view({column_view(nullptr, 0, I32)}), table_view({column_view(nullptr, 0, I64)}),
                                {{0, agg::SUM}}, ctx);
        if (e->num_rows() != 0 || e->num_columns() != 2) return 4;
        column_view l0(upload(pk), (size_type)pk.size(), I32), r0(upload(fk), (size_type)fk.size(), I32);
        auto j = phys::eq_join(table_view({l0}), {0}, table_view({r0}), {0}, ctx);
        if (j->num_columns() != 1) return 5;
        save_col("pjoin_key", j->get_column(0));
        auto f = phys::filter(table_view({kc, vc}), {select::predicate::on_int(1, select::cmp::LT, 500000)}, {0}, ctx);
        save_col("filter_key", f->get_column(0));
    }
    // pullops: Scan (batches of 100000) -> Filter (val < 500000) -> Aggregate (SUM by key)
    {
        std::vector<column_view> cols{kc, vc};
        table_view src(cols);
        auto scan = std::make_unique<pullops::Scan>(src, 100000);
        auto filt = std::make_unique<pullops::Filter>(
            std::move(scan), std::vector<select::predicate>{select::predicate::on_int(1, select::cmp::LT, 500000)});
        pullops::Aggregate aggop(std::move(filt), {0}, {1}, {{0, agg::SUM}});
        aggop.open();
        auto r = aggop.next();
        if (aggop.next() != nullptr) return 6;
        aggop.close();
        save_col("pull_key", r->get_column(0));
        save_col("pull_sum", r->get_column(1));
    }
    cudaDeviceSynchronize();
    std::printf("ok\n");
    return 0;
}
'''


def rd(d, name, dt):
    return np.fromfile(d / name, dtype=dt)


def test_reference_style_cpp_caller(tmp_path):
    n = 1 << 20
    key = O.gen_keys(n, np.int32, groups=5000, scatter=1, seed=1)
    key2 = O.gen_keys(n, np.int32, groups=7, seed=2)
    val = O.gen_values(n, np.int64, lo=0, hi=1_000_000, seed=3)
    pk = O.gen_perm(1 << 14, np.int32, seed=4)
    fk = O.gen_keys(1 << 17, np.int32, groups=1 << 14, seed=5, miss_frac=0.1)
    for nm, a in (("key", key), ("key2", key2), ("val", val), ("pk", pk), ("fk", fk)):
        a.tofile(tmp_path / f"{nm}.bin")
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", str(src), "-o",
                    str(exe), f"-L{ROOT / 'eiger_b200'}", "-lgx", f"-L{CUDA / 'lib64'}", "-lcudart",
                    f"-Wl,-rpath,{ROOT / 'eiger_b200'}", f"-Wl,-rpath,{CUDA / 'lib64'}"], check=True)
    res = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True)
    assert res.returncode == 0, (res.returncode, res.stdout, res.stderr)
    assert "table_encode:Cannot dictionary encode table" in res.stdout
    d = tmp_path

    ek, es, ec = O.groupby(key, [val], [(0, O.SUM), (0, O.COUNT_ALL)])
    for p in ("gb_hash_", "gb_part_"):
        k, s, c = rd(d, p + "key", np.int32), rd(d, p + "sum", np.int64), rd(d, p + "cnt", np.int64)
        o = np.argsort(k)
        assert np.array_equal(k[o], ek) and np.array_equal(s[o], es) and np.array_equal(c[o], ec)

    l, r = rd(d, "join_l", np.int64), rd(d, "join_r", np.int64)
    o = np.lexsort((r, l))
    el, er = O.join_pairs(pk, fk)
    assert np.array_equal(l[o], el) and np.array_equal(r[o], er)

    sk, sv = O.sort_pairs(key, val)
    assert np.array_equal(rd(d, "sort_k", np.int32), sk) and np.array_equal(rd(d, "sort_v", np.int64), sv)
    assert np.array_equal(rd(d, "part_off", np.int64), O.partition_offsets(sk, 0, 6))

    codes, nd = O.dict_encode(key, ordered=True)
    assert np.array_equal(rd(d, "dict_codes", np.int32), codes.astype(np.int32))
    assert f"ndv {nd}" in res.stdout

    assert rd(d, "agg_sum", np.int64)[0] == val.sum()
    assert rd(d, "agg_min", np.int64)[0] == val.min() and rd(d, "agg_max", np.int64)[0] == val.max()

    fused = key.astype(np.int64) * 8 + key2
    gk1, gk2 = rd(d, "mk_k1", np.int32), rd(d, "mk_k2", np.int32)
    _, fs, fc = O.groupby(fused, [val], [(0, O.SUM), (0, O.COUNT_ALL)])
    got = dict(zip(gk1.astype(np.int64) * 8 + gk2, zip(rd(d, "mk_sum", np.int64), rd(d, "mk_cnt", np.int64))))
    exp = dict(zip(np.unique(fused), zip(fs, fc)))
    assert got == exp

    assert np.array_equal(np.sort(rd(d, "distinct", np.int32)), np.unique(key))
    assert np.array_equal(np.sort(rd(d, "pjoin_key", np.int32)), np.sort(fk[np.isin(fk, pk)]))
    assert np.array_equal(rd(d, "filter_key", np.int32), key[val < 500000])

    keep = val < 500000
    pk_, ps_ = O.groupby(key[keep], [val[keep]], [(0, O.SUM)])
    k, s = rd(d, "pull_key", np.int32), rd(d, "pull_sum", np.int64)
    o = np.argsort(k)
    assert np.array_equal(k[o], pk_) and np.array_equal(s[o], ps_)
