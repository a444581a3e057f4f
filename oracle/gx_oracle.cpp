// gx_oracle.cpp — CPU oracle for the relational operator core.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the CPU, what the
// reference engine (BowenforGit/eiger, "GaMax", src/cuda/...) computes on the
// operator path, so the CUDA library can be checked against it.  It is used
// by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline /
// --impl reference arm, and by nothing in the product.
//
// Parity pinning: the reference ships no CPU implementation of these
// operators and its hash / partition / dictionary paths need cuCollections
// (not vendored), so the oracle is pinned against the reference's own test
// expectations instead (tests/golden/, produced by tests/golden/make_golden.py
// from src/cuda/tests/groupby/groupby_multikeys_test.cu, the closed forms of
// src/cuda/tests/groupby/groupby_test.hpp:64-92, the PK-FK counts of
// src/cuda/tests/join/ieq_join_test.cu:19-83, the dictionary checks of
// src/cuda/tests/compress/dictionary_encode_test.cu:16-52,160-202 and the
// partition checks of src/cuda/tests/sort/sort_partition_test.cu:16-42).
//
// Semantics restated (reference file:line):
//   * aggregation output types and identities: operators/groupby/agg_func.cuh:20-224,
//     operators/groupby/aggregate.cu:19-53;
//   * AVG = SUM / COUNT in double, COUNT_ALL / agg_count: operators/groupby/groupby.cu:29-50,128-244;
//   * radix digit of the order-preserving key image for sort / partition
//     (CUB DeviceRadixSort semantics behind operators/sort/sort.cu:15-66), stable;
//   * partition offsets = inclusive histogram scan over (key >> b) & mask:
//     operators/partition/partition.cu:103-149;
//   * merge-join match set = every (left, right) pair with equal keys:
//     operators/join/merge_path.cuh:155-184, output order [key, left.., right..]
//     operators/join/sort_merge_join.cu:183-206;
//   * dictionary encodings: compress/dictionary_encode.cu:71-142,
//     compress/dictionary_encode_dict_ready.cu:35-58 (absent value -> INT32_MIN).
// Group-by results are returned sorted by key (canonical order); float SUM
// accumulates in long double, in row order, so the oracle is closer to the
// exact sum than any device summation order.
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <parallel/algorithm>
#include <unordered_map>
#include <vector>

namespace {

enum { T_EMPTY, T_I8, T_I16, T_I32, T_I64, T_B8, T_U8, T_U16, T_U32, T_U64, T_F32, T_F64 };
enum { A_SUM, A_MAX, A_MIN, A_AVG, A_ANY, A_COUNT };

int width(int t) {
    switch (t) {
        case T_I8: case T_U8: case T_B8: return 1;
        case T_I16: case T_U16: return 2;
        case T_I32: case T_U32: case T_F32: return 4;
        case T_I64: case T_U64: case T_F64: return 8;
    }
    return 0;
}
bool is_f(int t) { return t == T_F32 || t == T_F64; }
bool is_s(int t) { return t == T_I8 || t == T_I16 || t == T_I32 || t == T_I64; }

uint64_t raw_bits(const void* p, int t, int64_t i) {
    switch (width(t)) {
        case 1: return ((const uint8_t*)p)[i];
        case 2: return ((const uint16_t*)p)[i];
        case 4: return ((const uint32_t*)p)[i];
        default: return ((const uint64_t*)p)[i];
    }
}
// Canonical equality bits (float -0.0 == +0.0).
uint64_t canon(uint64_t b, int t) {
    if (t == T_F32 && (uint32_t)(b << 1) == 0) return 0;
    if (t == T_F64 && (b << 1) == 0) return 0;
    return b;
}
// Order-preserving image in the key's own width.
uint64_t image(uint64_t b, int t) {
    int w = width(t);
    if (is_s(t)) return b ^ (1ull << (8 * w - 1));
    if (t == T_F32) {
        uint32_t x = (uint32_t)b;
        if (x == 0x80000000u) x = 0;
        return (x & 0x80000000u) ? (uint32_t)~x : (x | 0x80000000u);
    }
    if (t == T_F64) {
        if (b == 0x8000000000000000ull) b = 0;
        return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
    }
    return b;
}

long double as_ld(const void* p, int t, int64_t i) {
    switch (t) {
        case T_I8: return ((const int8_t*)p)[i];
        case T_I16: return ((const int16_t*)p)[i];
        case T_I32: return ((const int32_t*)p)[i];
        case T_I64: return (long double)((const int64_t*)p)[i];
        case T_U8: case T_B8: return ((const uint8_t*)p)[i];
        case T_U16: return ((const uint16_t*)p)[i];
        case T_U32: return ((const uint32_t*)p)[i];
        case T_U64: return (long double)((const uint64_t*)p)[i];
        case T_F32: return ((const float*)p)[i];
        default: return ((const double*)p)[i];
    }
}
int64_t as_i64(const void* p, int t, int64_t i) {
    switch (t) {
        case T_I8: return ((const int8_t*)p)[i];
        case T_I16: return ((const int16_t*)p)[i];
        case T_I32: return ((const int32_t*)p)[i];
        case T_I64: return ((const int64_t*)p)[i];
        default: return (int64_t)raw_bits(p, t, i);  // unsigned: zero-extended
    }
}

// Per-group accumulator of one value column: integer sums wrap in uint64,
// float sums accumulate in long double; mn / mx hold the extreme's bits
// (int64 / uint64 value, or the double for float columns); NaN does not take
// part in MIN / MAX, and a group with no non-NaN value keeps seen = false.
struct cacc {
    long double fsum;
    uint64_t isum;
    uint64_t mn, mx;
    uint64_t any;
    bool seen;
};

void cacc_init(cacc& x, uint64_t any_bits) {
    x.fsum = 0;
    x.isum = 0;
    x.mn = x.mx = 0;
    x.any = any_bits;
    x.seen = false;
}

void cacc_update(cacc& x, const void* col, int t, int64_t i) {
    if (is_f(t)) {
        const double v = t == T_F32 ? (double)((const float*)col)[i] : ((const double*)col)[i];
        x.fsum += (long double)v;
        if (std::isnan(v)) return;
        uint64_t b;
        memcpy(&b, &v, 8);
        if (!x.seen) { x.mn = x.mx = b; x.seen = true; return; }
        double mn, mx;
        memcpy(&mn, &x.mn, 8);
        memcpy(&mx, &x.mx, 8);
        if (v < mn) x.mn = b;
        if (v > mx) x.mx = b;
    } else if (is_s(t)) {
        const int64_t v = as_i64(col, t, i);
        x.isum += (uint64_t)v;
        if (!x.seen) { x.mn = x.mx = (uint64_t)v; x.seen = true; return; }
        if (v < (int64_t)x.mn) x.mn = (uint64_t)v;
        if (v > (int64_t)x.mx) x.mx = (uint64_t)v;
    } else {
        const uint64_t v = raw_bits(col, t, i);
        x.isum += v;
        if (!x.seen) { x.mn = x.mx = v; x.seen = true; return; }
        if (v < x.mn) x.mn = v;
        if (v > x.mx) x.mx = v;
    }
}

uint64_t o_fmix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}
int ceil_log2(uint64_t x) { int b = 0; while ((1ull << b) < x) ++b; return b; }

int out_type(int kind, int t) {
    if (kind == A_COUNT) return T_I64;
    if (kind == A_AVG) return T_F64;
    if (kind == A_SUM) {
        if (is_f(t)) return t;
        return is_s(t) ? T_I64 : T_U64;
    }
    return t;
}

void store(void* out, int t, int64_t i, uint64_t bits_or_int, long double fv, bool use_f) {
    switch (t) {
        case T_I8: ((int8_t*)out)[i] = (int8_t)bits_or_int; break;
        case T_U8: case T_B8: ((uint8_t*)out)[i] = (uint8_t)bits_or_int; break;
        case T_I16: ((int16_t*)out)[i] = (int16_t)bits_or_int; break;
        case T_U16: ((uint16_t*)out)[i] = (uint16_t)bits_or_int; break;
        case T_I32: ((int32_t*)out)[i] = (int32_t)bits_or_int; break;
        case T_U32: ((uint32_t*)out)[i] = (uint32_t)bits_or_int; break;
        case T_F32: ((float*)out)[i] = use_f ? (float)fv : (float)fv; break;
        case T_F64: ((double*)out)[i] = (double)fv; break;
        default: ((uint64_t*)out)[i] = bits_or_int; break;
    }
}

}  // namespace

extern "C" {

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// ---------------------------------------------------------------------------
// Group-by.  vals[c] / val_types[c]: value columns; requests (col, kind);
// outputs: out_key (capacity n, key type), out[r] (capacity n, output type of
// request r; when agg_count an extra trailing int64 count column).
// Returns the number of groups, sorted ascending by key.
//
// Method (also the timed CPU baseline): radix-partition the row ids by the
// top bits of a 64-bit key hash (per-thread counts, prefix, stable scatter, so
// each partition keeps row order), then aggregate every partition with its
// own open-addressing table, partitions spread over the threads.  Partitions
// hold disjoint keys, so nothing is merged; each group sees its rows in row
// order, which fixes ANY (first row) and the long double float sums.
// ---------------------------------------------------------------------------
int64_t orc_groupby(const void* keys, int key_type, int64_t n, int nvals, const void* const* vals,
                    const int* val_types, int nreq, const int64_t* req_cols, const int* req_kinds,
                    int agg_count, void* out_key, void* const* out) {
    if ((uint64_t)n >= (1ull << 32)) return -1;
    const int T = omp_get_max_threads();
    int pb = 0;
    if (n >= (1 << 16)) pb = std::min(12, ceil_log2((uint64_t)n >> 15));
    const int64_t P = int64_t(1) << pb;
    auto khash = [&](uint64_t k) { return o_fmix64(k ^ 0x9E3779B97F4A7C15ull); };
    auto part_of = [&](int64_t i) -> int64_t {
        return pb ? (int64_t)(khash(canon(raw_bits(keys, key_type, i), key_type)) >> (64 - pb)) : 0;
    };
    std::vector<int64_t> cnt((size_t)T * P, 0), off((size_t)T * P, 0), start(P + 1, 0);
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const int64_t lo = n * t / T, hi = n * (t + 1) / T;
        int64_t* c = &cnt[(size_t)t * P];
        for (int64_t i = lo; i < hi; ++i) c[part_of(i)]++;
    }
    int64_t run = 0;
    for (int64_t p = 0; p < P; ++p) {
        start[p] = run;
        for (int t = 0; t < T; ++t) { off[(size_t)t * P + p] = run; run += cnt[(size_t)t * P + p]; }
    }
    start[P] = run;
    std::vector<uint32_t> idx((size_t)n);
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const int64_t lo = n * t / T, hi = n * (t + 1) / T;
        int64_t* o = &off[(size_t)t * P];
        for (int64_t i = lo; i < hi; ++i) idx[(size_t)o[part_of(i)]++] = (uint32_t)i;
    }
    struct part_out {
        std::vector<uint64_t> key_raw;
        std::vector<int64_t> count;
        std::vector<cacc> a;  // nvals per group
    };
    std::vector<part_out> po((size_t)P);
    // Per-thread working table and group lists, reused from partition to
    // partition (growing vectors per partition costs fresh pages and unmaps
    // on every growth step); each partition's groups are copied out once.
    std::vector<part_out> work((size_t)T);
    std::vector<std::vector<uint64_t>> wtk((size_t)T);
    std::vector<std::vector<int32_t>> wtg((size_t)T);
#pragma omp parallel for schedule(dynamic, 1) num_threads(T)
    for (int64_t p = 0; p < P; ++p) {
        const int t = omp_get_thread_num();
        part_out& o = work[(size_t)t];
        std::vector<uint64_t>& tk = wtk[(size_t)t];
        std::vector<int32_t>& tg = wtg[(size_t)t];
        o.key_raw.clear();
        o.count.clear();
        o.a.clear();
        uint64_t cap = 1024;
        if (tk.size() < cap) { tk.resize(cap); tg.resize(cap); }
        std::fill(tg.begin(), tg.begin() + (int64_t)cap, -1);
        for (int64_t j = start[p]; j < start[p + 1]; ++j) {
            const int64_t i = idx[(size_t)j];
            const uint64_t raw = raw_bits(keys, key_type, i), k = canon(raw, key_type);
            uint64_t slot = khash(k) & (cap - 1);
            int32_t g;
            for (;;) {
                if (tg[slot] < 0) {
                    g = (int32_t)o.count.size();
                    tg[slot] = g;
                    tk[slot] = k;
                    o.key_raw.push_back(raw);
                    o.count.push_back(0);
                    for (int c = 0; c < nvals; ++c) {
                        cacc x;
                        cacc_init(x, raw_bits(vals[c], val_types[c], i));
                        o.a.push_back(x);
                    }
                    if ((uint64_t)o.count.size() * 2 > cap) {  // keep load <= 1/2: rebuild at twice the size
                        cap *= 2;
                        if (tk.size() < cap) { tk.resize(cap); tg.resize(cap); }
                        std::fill(tg.begin(), tg.begin() + (int64_t)cap, -1);
                        for (size_t q = 0; q < o.count.size(); ++q) {
                            const uint64_t kq = canon(o.key_raw[q], key_type);
                            uint64_t sq = khash(kq) & (cap - 1);
                            while (tg[sq] >= 0) sq = (sq + 1) & (cap - 1);
                            tg[sq] = (int32_t)q;
                            tk[sq] = kq;
                        }
                    }
                    break;
                }
                if (tk[slot] == k) { g = tg[slot]; break; }
                slot = (slot + 1) & (cap - 1);
            }
            o.count[(size_t)g]++;
            for (int c = 0; c < nvals; ++c) cacc_update(o.a[(size_t)g * nvals + c], vals[c], val_types[c], i);
        }
        part_out& dst = po[(size_t)p];
        dst.key_raw.assign(o.key_raw.begin(), o.key_raw.end());
        dst.count.assign(o.count.begin(), o.count.end());
        dst.a.assign(o.a.begin(), o.a.end());
    }
    // Canonical order: ascending key image.
    struct gref { uint64_t img; uint32_t p, g; };
    std::vector<int64_t> gstart(P + 1, 0);
    for (int64_t p = 0; p < P; ++p) gstart[p + 1] = gstart[p] + (int64_t)po[(size_t)p].count.size();
    const int64_t G = gstart[P];
    std::vector<gref> order((size_t)G);
#pragma omp parallel for schedule(dynamic, 16) num_threads(T)
    for (int64_t p = 0; p < P; ++p)
        for (size_t g = 0; g < po[(size_t)p].count.size(); ++g)
            order[(size_t)(gstart[p] + (int64_t)g)] = {image(canon(po[(size_t)p].key_raw[g], key_type), key_type),
                                                       (uint32_t)p, (uint32_t)g};
    __gnu_parallel::sort(order.begin(), order.end(), [](const gref& x, const gref& y) { return x.img < y.img; });
    const int kw = width(key_type);
#pragma omp parallel for schedule(static) num_threads(T)
    for (int64_t gi = 0; gi < G; ++gi) {
        const part_out& o = po[order[(size_t)gi].p];
        const size_t g = order[(size_t)gi].g;
        const int64_t count = o.count[g];
        memcpy((char*)out_key + gi * kw, &o.key_raw[g], kw);
        for (int r = 0; r < nreq; ++r) {
            const int kind = req_kinds[r];
            if (kind == A_COUNT) { ((int64_t*)out[r])[gi] = count; continue; }
            const int c = (int)req_cols[r];
            const int t = val_types[c];
            const cacc& x = o.a[g * nvals + c];
            const int ot = out_type(kind, t);
            switch (kind) {
                case A_SUM:
                    if (is_f(t)) store(out[r], ot, gi, 0, x.fsum, true);
                    else store(out[r], ot, gi, x.isum, 0, false);
                    break;
                case A_AVG: {
                    long double num = is_f(t) ? x.fsum : (is_s(t) ? (long double)(int64_t)x.isum : (long double)x.isum);
                    ((double*)out[r])[gi] = (double)(num / (long double)count);
                    break;
                }
                case A_MIN: case A_MAX: {
                    const uint64_t b = kind == A_MIN ? x.mn : x.mx;
                    if (is_f(t)) {
                        double d = 0;
                        if (x.seen) memcpy(&d, &b, 8);
                        store(out[r], ot, gi, 0, (long double)d, true);
                    } else {
                        store(out[r], ot, gi, x.seen ? b : 0, 0, false);
                    }
                    break;
                }
                case A_ANY: {
                    int w = width(t);
                    memcpy((char*)out[r] + gi * w, &x.any, w);
                    break;
                }
            }
        }
        if (agg_count) ((int64_t*)out[nreq])[gi] = count;
    }
    return G;
}

// ---------------------------------------------------------------------------
// Stable sort / partition on bits [b, e) of the key image.
// vals may be null; when iota the values are row ids (int64).
// ---------------------------------------------------------------------------
void orc_sort_pairs(const void* keys, int key_type, int64_t n, const void* vals, int val_width, int iota, int b,
                    int e, int desc, void* out_keys, void* out_vals) {
    int kw = width(key_type);
    if (e <= 0 || e > 8 * kw) e = 8 * kw;
    if (b < 0) b = 0;
    uint64_t mask = (e - b) >= 64 ? ~0ull : ((1ull << (e - b)) - 1);
    std::vector<uint64_t> dig(n);
    uint64_t allbits = kw == 8 ? ~0ull : ((1ull << (8 * kw)) - 1);
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        uint64_t img = image(raw_bits(keys, key_type, i), key_type);
        if (desc) img = (~img) & allbits;
        dig[i] = b >= 64 ? 0 : (img >> b) & mask;
    }
    std::vector<int64_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) { return dig[x] < dig[y]; });
    if (iota) val_width = 8;
    for (int64_t i = 0; i < n; ++i) {
        memcpy((char*)out_keys + i * kw, (const char*)keys + idx[i] * kw, kw);
        if (out_vals) {
            if (iota) ((int64_t*)out_vals)[i] = idx[i];
            else if (vals && val_width) memcpy((char*)out_vals + i * val_width, (const char*)vals + idx[i] * val_width, val_width);
        }
    }
}

// Inclusive offsets, P+1 entries, last = n (digit on the raw key value).
void orc_partition_offsets(const void* keys, int key_type, int64_t n, int b, int e, int64_t* out) {
    int64_t P = 1ll << (e - b);
    std::vector<int64_t> h(P, 0);
    for (int64_t i = 0; i < n; ++i) h[(raw_bits(keys, key_type, i) >> b) & (P - 1)]++;
    int64_t run = 0;
    for (int64_t p = 0; p < P; ++p) { run += h[p]; out[p] = run; }
    out[P] = n;
}

// ---------------------------------------------------------------------------
// Inner equi-join: all (left_row, right_row) with equal keys, sorted by
// (left_row, right_row).  Call with out_l == null to get the count.
// ---------------------------------------------------------------------------
int64_t orc_join_pairs(const void* lkeys, int64_t nl, const void* rkeys, int64_t nr, int key_type, int64_t* out_l,
                       int64_t* out_r) {
    std::unordered_map<uint64_t, std::vector<int64_t>> idx;
    idx.reserve((size_t)nl * 2 + 1);
    for (int64_t i = 0; i < nl; ++i) idx[canon(raw_bits(lkeys, key_type, i), key_type)].push_back(i);
    // Count per right row, then emit grouped by left row order via sort.
    std::vector<std::pair<int64_t, int64_t>> pairs;
    int64_t total = 0;
    for (int64_t j = 0; j < nr; ++j) {
        auto it = idx.find(canon(raw_bits(rkeys, key_type, j), key_type));
        if (it == idx.end()) continue;
        total += (int64_t)it->second.size();
        if (out_l)
            for (int64_t i : it->second) pairs.emplace_back(i, j);
    }
    if (!out_l) return total;
    std::sort(pairs.begin(), pairs.end());
    for (size_t k = 0; k < pairs.size(); ++k) { out_l[k] = pairs[k].first; out_r[k] = pairs[k].second; }
    return total;
}

// Parallel count-only probe (for timing the CPU baseline on large inputs):
// hash build of the left side, probe of the right side.
int64_t orc_join_count_parallel(const void* lkeys, int64_t nl, const void* rkeys, int64_t nr, int key_type) {
    std::unordered_map<uint64_t, int64_t> cnt;
    cnt.reserve((size_t)nl * 2 + 1);
    for (int64_t i = 0; i < nl; ++i) cnt[canon(raw_bits(lkeys, key_type, i), key_type)]++;
    int64_t total = 0;
#pragma omp parallel for reduction(+ : total)
    for (int64_t j = 0; j < nr; ++j) {
        auto it = cnt.find(canon(raw_bits(rkeys, key_type, j), key_type));
        if (it != cnt.end()) total += it->second;
    }
    return total;
}

// Unique-build probe: match[j] = the left row whose key equals right row j's,
// or -1.  Returns 0, or -1 when the left keys are not unique (match is then
// unspecified).  Every (left, right) pair of the join is (match[j], j) for
// match[j] >= 0, so this checks a join of a unique build side in O(n).
int64_t orc_join_probe_unique(const void* lkeys, int64_t nl, const void* rkeys, int64_t nr, int key_type,
                              int64_t* match) {
    const uint64_t cap = 1ull << ceil_log2((uint64_t)std::max<int64_t>(2 * nl, 2));
    std::vector<uint64_t> tk(cap);
    std::vector<int64_t> tr(cap, -1);
    for (int64_t i = 0; i < nl; ++i) {
        const uint64_t k = canon(raw_bits(lkeys, key_type, i), key_type);
        uint64_t s = o_fmix64(k) & (cap - 1);
        while (tr[s] >= 0) {
            if (tk[s] == k) return -1;
            s = (s + 1) & (cap - 1);
        }
        tk[s] = k;
        tr[s] = i;
    }
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < nr; ++j) {
        const uint64_t k = canon(raw_bits(rkeys, key_type, j), key_type);
        uint64_t s = o_fmix64(k) & (cap - 1);
        int64_t m = -1;
        while (tr[s] >= 0) {
            if (tk[s] == k) { m = tr[s]; break; }
            s = (s + 1) & (cap - 1);
        }
        match[j] = m;
    }
    return 0;
}

// Parallel hash join (the timed CPU join baseline): chained table over the
// left keys, right rows probed by all threads; pairs are written in right-row
// order, each right row's matches in descending left row order.  Call with
// out_l == null for the count only.
int64_t orc_join_pairs_parallel(const void* lkeys, int64_t nl, const void* rkeys, int64_t nr, int key_type,
                                int64_t* out_l, int64_t* out_r) {
    const uint64_t cap = 1ull << ceil_log2((uint64_t)std::max<int64_t>(nl, 2));
    std::vector<int64_t> head(cap, -1), next((size_t)std::max<int64_t>(nl, 1));
    std::vector<uint64_t> lk((size_t)std::max<int64_t>(nl, 1));
    for (int64_t i = 0; i < nl; ++i) {
        const uint64_t k = canon(raw_bits(lkeys, key_type, i), key_type);
        const uint64_t s = o_fmix64(k) & (cap - 1);
        lk[i] = k;
        next[i] = head[s];
        head[s] = i;
    }
    const int T = omp_get_max_threads();
    std::vector<int64_t> part(T + 1, 0);
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const int64_t lo = nr * t / T, hi = nr * (t + 1) / T;
        int64_t c = 0;
        for (int64_t j = lo; j < hi; ++j) {
            const uint64_t k = canon(raw_bits(rkeys, key_type, j), key_type);
            for (int64_t i = head[o_fmix64(k) & (cap - 1)]; i >= 0; i = next[i]) c += lk[i] == k;
        }
        part[t + 1] = c;
#pragma omp barrier
#pragma omp single
        for (int q = 0; q < T; ++q) part[q + 1] += part[q];
        if (out_l) {
            int64_t w = part[t];
            for (int64_t j = lo; j < hi; ++j) {
                const uint64_t k = canon(raw_bits(rkeys, key_type, j), key_type);
                for (int64_t i = head[o_fmix64(k) & (cap - 1)]; i >= 0; i = next[i])
                    if (lk[i] == k) { out_l[w] = i; out_r[w] = j; ++w; }
            }
        }
    }
    return part[T];
}

// ---------------------------------------------------------------------------
// Dictionary encoding.  mode 0: codes in first-occurrence order; mode 1:
// code = rank of the value among distinct values.  Returns NDV.
// ---------------------------------------------------------------------------
int64_t orc_dict_encode(const void* keys, int key_type, int64_t n, int mode, int64_t* codes) {
    std::unordered_map<uint64_t, int64_t> m;
    std::vector<uint64_t> firsts;
    for (int64_t i = 0; i < n; ++i) {
        uint64_t k = canon(raw_bits(keys, key_type, i), key_type);
        auto it = m.find(k);
        if (it == m.end()) {
            int64_t c = (int64_t)firsts.size();
            m.emplace(k, c);
            firsts.push_back(k);
            codes[i] = c;
        } else {
            codes[i] = it->second;
        }
    }
    if (mode == 1) {
        std::vector<int64_t> ord(firsts.size());
        std::iota(ord.begin(), ord.end(), 0);
        std::sort(ord.begin(), ord.end(), [&](int64_t x, int64_t y) { return image(firsts[x], key_type) < image(firsts[y], key_type); });
        std::vector<int64_t> rank(firsts.size());
        for (size_t r = 0; r < ord.size(); ++r) rank[ord[r]] = (int64_t)r;
        for (int64_t i = 0; i < n; ++i) codes[i] = rank[codes[i]];
    }
    return (int64_t)firsts.size();
}

// Ready dictionary: position (smallest for duplicates), INT32_MIN if absent.
void orc_dict_with_dict(const void* keys, int64_t n, const void* dict, int64_t nd, int key_type, int32_t* out) {
    std::unordered_map<uint64_t, int64_t> pos;
    for (int64_t i = nd - 1; i >= 0; --i) pos[canon(raw_bits(dict, key_type, i), key_type)] = i;
    for (int64_t i = 0; i < n; ++i) {
        auto it = pos.find(canon(raw_bits(keys, key_type, i), key_type));
        out[i] = it == pos.end() ? std::numeric_limits<int32_t>::min() : (int32_t)it->second;
    }
}

int64_t orc_ndv_exact(const void* keys, int key_type, int64_t n) {
    std::vector<uint64_t> v(n);
    for (int64_t i = 0; i < n; ++i) v[i] = canon(raw_bits(keys, key_type, i), key_type);
    std::sort(v.begin(), v.end());
    return (int64_t)(std::unique(v.begin(), v.end()) - v.begin());
}

// ---------------------------------------------------------------------------
// HyperLogLog (p = 13) restated from Flajolet et al. 2007 with the same hash
// and register rule as the device sketch, so registers match bit for bit.
// ---------------------------------------------------------------------------
void orc_hll_registers(const void* keys, int key_type, int64_t n, int64_t stride, uint32_t* regs) {
    const int P = 13;
    memset(regs, 0, sizeof(uint32_t) << P);
    for (int64_t j = 0; j < n; ++j) {
        uint64_t b = canon(raw_bits(keys, key_type, j * stride), key_type);
        uint64_t h = o_fmix64(b ^ 0x5bd1e9955bd1e995ull);
        uint32_t idx = (uint32_t)(h >> (64 - P));
        uint64_t w = (h << P) | (1ull << (P - 1));
        uint32_t rank = (uint32_t)__builtin_clzll(w) + 1;
        if (regs[idx] < rank) regs[idx] = rank;
    }
}
double orc_hll_estimate(const uint32_t* regs) {
    const int M = 1 << 13;
    double m = M, alpha = 0.7213 / (1.0 + 1.079 / m), sum = 0;
    int zeros = 0;
    for (int i = 0; i < M; ++i) { sum += std::ldexp(1.0, -(int)regs[i]); zeros += regs[i] == 0; }
    double e = alpha * m * m / sum;
    if (e <= 2.5 * m && zeros > 0) e = m * std::log(m / zeros);
    return e;
}

// ---------------------------------------------------------------------------
// Generators: the same SplitMix64 counter construction as the device
// generator (restated independently so the tests compare the two).
// ---------------------------------------------------------------------------
static uint64_t sm_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t sm_base(uint64_t seed, uint64_t sid) { return sm_mix(seed ^ sm_mix(sid + 0xD1B54A32D192ED03ull)); }
static uint64_t sm_at(uint64_t base, uint64_t i) { return sm_mix(base + (i + 1) * 0x9E3779B97F4A7C15ull); }
static uint64_t mulhi(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) >> 64); }
static uint64_t perm_bits(uint64_t x, int k, uint64_t key) {
    if (k == 0) return 0;
    uint64_t mask = k >= 64 ? ~0ull : ((1ull << k) - 1);
    int sh = k / 2 + 1;
    for (int r = 0; r < 4; ++r) {
        uint64_t rk = sm_mix(key + r);
        x = (x + rk) & mask;
        x = (x * (rk | 1ull)) & mask;
        x ^= (sh < 64 ? (x >> sh) : 0);
    }
    return x;
}
static uint64_t perm_range(uint64_t i, uint64_t n, int k, uint64_t key) {
    uint64_t x = i;
    do { x = perm_bits(x, k, key); } while (x >= n);
    return x;
}
static uint32_t o_fmix32(uint32_t x) {
    x ^= x >> 16; x *= 0x85ebca6bU; x ^= x >> 13; x *= 0xc2b2ae35U; x ^= x >> 16;
    return x;
}

void orc_zipf_cdf(int64_t G, double s, double* cdf) {
    double total = 0.0;
    for (int64_t r = 0; r < G; ++r) { total += 1.0 / std::pow((double)(r + 1), s); cdf[r] = total; }
    for (int64_t r = 0; r < G; ++r) cdf[r] /= total;
    if (G > 0) cdf[G - 1] = 1.0;
}

// dist: 0 uniform, 1 cyclic (shuffled i % G), 2 zipf (cdf), 3 sequence.
void orc_gen_keys(void* out, int64_t n, int w, uint64_t seed, uint64_t sid, int dist, int scatter, int64_t groups,
                  const double* cdf, double miss_frac) {
    uint64_t base = sm_base(seed, sid), G = groups > 0 ? (uint64_t)groups : 1;
    uint64_t mbase = sm_base(seed, sid ^ 0x6D15ull);
    uint64_t thr = miss_frac > 0 ? (uint64_t)(miss_frac * 0x1.0p53) : 0;
    int k = ceil_log2((uint64_t)n);
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        uint64_t r;
        uint64_t m = thr ? sm_at(mbase, (uint64_t)i) : 0;
        if (thr && (m >> 11) < thr) r = G + mulhi(sm_mix(m), G);
        else if (dist == 1) r = perm_range((uint64_t)i, (uint64_t)n, k, seed ^ 0xA5A5A5A5ull) % G;
        else if (dist == 2) {
            double u = (double)(sm_at(base, (uint64_t)i) >> 11) * 0x1.0p-53;
            int64_t lo = 0, hi = (int64_t)G;
            while (lo < hi) { int64_t mid = lo + (hi - lo) / 2; if (cdf[mid] <= u) lo = mid + 1; else hi = mid; }
            r = (uint64_t)(lo < (int64_t)G ? lo : (int64_t)G - 1);
        } else if (dist == 3) r = (uint64_t)i;
        else r = mulhi(sm_at(base, (uint64_t)i), G);
        if (w == 4) ((uint32_t*)out)[i] = scatter ? o_fmix32((uint32_t)r ^ 0x5bd1e995u) : (uint32_t)r;
        else ((uint64_t*)out)[i] = scatter ? o_fmix64(r ^ 0x5bd1e9955bd1e995ull) : r;
    }
}

void orc_gen_values(void* out, int64_t n, int type, uint64_t seed, uint64_t sid, int64_t lo, int64_t hi) {
    uint64_t base = sm_base(seed, sid), span = (uint64_t)(hi - lo);
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        uint64_t r = sm_at(base, (uint64_t)i);
        switch (type) {
            case T_F64: ((double*)out)[i] = (double)(r >> 11) * 0x1.0p-53; break;
            case T_F32: ((float*)out)[i] = (float)(r >> 40) * 0x1.0p-24f; break;
            case T_I64: case T_U64: ((int64_t*)out)[i] = lo + (int64_t)mulhi(r, span); break;
            case T_I32: case T_U32: ((int32_t*)out)[i] = (int32_t)(lo + (int64_t)mulhi(r, span)); break;
            case T_I16: case T_U16: ((int16_t*)out)[i] = (int16_t)(lo + (int64_t)mulhi(r, span)); break;
            default: ((int8_t*)out)[i] = (int8_t)(lo + (int64_t)mulhi(r, span)); break;
        }
    }
}

void orc_gen_perm(void* out, int64_t n, int w, uint64_t seed, int64_t base_v) {
    int k = ceil_log2((uint64_t)n);
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        int64_t v = (int64_t)perm_range((uint64_t)i, (uint64_t)n, k, seed) + base_v;
        if (w == 4) ((int32_t*)out)[i] = (int32_t)v;
        else ((int64_t*)out)[i] = v;
    }
}

}  // extern "C"
