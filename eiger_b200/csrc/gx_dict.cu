// gx_dict.cu — dictionary encoding.
//
// Replaces gamax::compress::dictionary_encode{,_with_order} and the
// ready-dictionary overload (src/cuda/compress/dictionary_encode.cu:144-373,
// src/cuda/compress/dictionary_encode_dict_ready.cu:16-82).  The reference
// inserts row ids into a cuco set sized N/0.25 when no hint is given, writes
// an int64 representative per row and gathers codes through it.  Here the
// table holds the canonical key bits and their code directly:
//   * hash encode: pass 1 inserts keys and hands each new key the next code
//     (atomicAdd); pass 2 looks every row up and writes its code — no
//     per-row int64 scratch;
//   * order-preserving: pass 1 inserts keys, the distinct keys are compacted
//     and radix-sorted, each key's slot receives its rank, pass 2 as above;
//   * ready dictionary: the dictionary's values are inserted with code =
//     position (the smallest position wins for duplicated values); rows whose
//     value is absent get INT32_MIN (gamax::sentinel<int32_t>()).
// Without a size hint the table is sized from a HyperLogLog estimate
// instead of the row count.
#include <algorithm>
#include <cmath>

#include "gx_groupby.h"

namespace gx {
namespace {

constexpr uint64_t D_EMPTY4 = ~0ull;
constexpr uint64_t D_EMPTY8 = 0x8000000000000000ull;
constexpr uint64_t NO_CODE = ~0ull;

struct dtable {
    unsigned long long* keys;   // cap + 1 slots; slot cap = key equal to the empty marker
    unsigned long long* codes;  // cap + 1
    uint64_t mask;
    int* overflow;
};

template <int KW>
__device__ __forceinline__ uint64_t dkey(const void* p, int64_t i, int kind) {
    if (KW == 4) return canon32(__ldg(static_cast<const unsigned*>(p) + i), kind);
    return canon64(__ldg(static_cast<const unsigned long long*>(p) + i), kind);
}
template <int KW>
__device__ __forceinline__ uint64_t dhash(uint64_t k) {
    if (KW == 4) return fmix32((uint32_t)k);
    return fmix64(k);
}

// Returns the slot index, inserting when `insert`; -1 when absent / overflow.
template <int KW>
__device__ __forceinline__ int64_t d_find(const dtable& t, uint64_t k, bool insert, bool* inserted) {
    const uint64_t EMPTY = KW == 4 ? D_EMPTY4 : D_EMPTY8;
    *inserted = false;
    if (KW == 8 && k == EMPTY) {
        int64_t s = (int64_t)t.mask + 1;
        if (insert) {
            unsigned long long old = atomicCAS(&t.keys[s], (unsigned long long)EMPTY ^ 1ull, (unsigned long long)EMPTY);
            *inserted = old == (EMPTY ^ 1ull);
            return s;
        }
        return t.keys[s] == EMPTY ? s : -1;
    }
    uint64_t slot = dhash<KW>(k) & t.mask;
    for (uint64_t p = 0, lim = t.mask < GX_PROBE_LIMIT ? t.mask : GX_PROBE_LIMIT - 1; p <= lim; ++p) {
        unsigned long long cur = ((volatile unsigned long long*)t.keys)[slot];
        if (cur == k) return (int64_t)slot;
        if (cur == EMPTY) {
            if (!insert) return -1;
            unsigned long long old = atomicCAS(&t.keys[slot], (unsigned long long)EMPTY, (unsigned long long)k);
            if (old == EMPTY) { *inserted = true; return (int64_t)slot; }
            if (old == k) return (int64_t)slot;
        }
        slot = (slot + 1) & t.mask;
    }
    if (insert) atomicExch(t.overflow, 1);
    return -1;
}

// Rows per thread per round of the insert and lookup kernels: their keys are
// loaded, then their home slots probed, all at once, so each thread keeps
// DU independent table reads in flight instead of one dependent chain.
constexpr int DU = 4;

// Slot of key k when it sits in its home slot (one plain load), else -1.
// A stale read (the key being inserted by another thread) only sends the
// row to the full probe walk.
template <int KW>
__device__ __forceinline__ int64_t d_home(const dtable& t, uint64_t k) {
    if (KW == 8 && k == D_EMPTY8) return -1;
    const uint64_t slot = dhash<KW>(k) & t.mask;
    return t.keys[slot] == k ? (int64_t)slot : -1;
}

template <int KW>
__global__ void k_dict_insert(const void* __restrict__ keys, int64_t n, int kind, dtable t, int assign,
                              unsigned long long* __restrict__ counter) {
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i0 < n; i0 += step * DU) {
        uint64_t k[DU];
        int64_t home[DU];
#pragma unroll
        for (int q = 0; q < DU; ++q) k[q] = i0 + q * step < n ? dkey<KW>(keys, i0 + q * step, kind) : 0;
#pragma unroll
        for (int q = 0; q < DU; ++q) home[q] = i0 + q * step < n ? d_home<KW>(t, k[q]) : 0;
#pragma unroll
        for (int q = 0; q < DU; ++q) {
            if (i0 + q * step >= n || home[q] >= 0) continue;
            bool ins;
            int64_t s = d_find<KW>(t, k[q], true, &ins);
            if (ins) {
                unsigned long long c = atomicAdd(counter, 1ull);
                if (assign) t.codes[s] = c;
            }
        }
    }
}

// Ready dictionary: insert value -> smallest position.
template <int KW>
__global__ void k_dict_insert_positions(const void* __restrict__ dict, int64_t n, int kind, dtable t) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        bool ins;
        int64_t s = d_find<KW>(t, dkey<KW>(dict, i, kind), true, &ins);
        if (s >= 0) atomicMin(&t.codes[s], (unsigned long long)i);
    }
}

__device__ __forceinline__ void store_code(void* out, int w, int64_t i, uint64_t c) {
    switch (w) {
        case 8: static_cast<unsigned long long*>(out)[i] = c; break;
        case 4: static_cast<unsigned*>(out)[i] = (unsigned)c; break;
        case 2: static_cast<uint16_t*>(out)[i] = (uint16_t)c; break;
        default: static_cast<uint8_t*>(out)[i] = (uint8_t)c; break;
    }
}

template <int KW>
__global__ void k_dict_lookup(const void* __restrict__ keys, int64_t n, int kind, dtable t, void* out, int ow,
                              uint64_t missing) {
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i0 < n; i0 += step * DU) {
        uint64_t k[DU];
        int64_t slot[DU];
#pragma unroll
        for (int q = 0; q < DU; ++q) k[q] = i0 + q * step < n ? dkey<KW>(keys, i0 + q * step, kind) : 0;
#pragma unroll
        for (int q = 0; q < DU; ++q) slot[q] = i0 + q * step < n ? d_home<KW>(t, k[q]) : 0;
#pragma unroll
        for (int q = 0; q < DU; ++q) {
            if (i0 + q * step >= n || slot[q] >= 0) continue;
            bool ins;
            slot[q] = d_find<KW>(t, k[q], false, &ins);
        }
        uint64_t c[DU];
#pragma unroll
        for (int q = 0; q < DU; ++q) c[q] = i0 + q * step < n && slot[q] >= 0 ? t.codes[slot[q]] : NO_CODE;
#pragma unroll
        for (int q = 0; q < DU; ++q)
            if (i0 + q * step < n) store_code(out, ow, i0 + q * step, c[q] == NO_CODE ? missing : c[q]);
    }
}

// Compact occupied slots' keys (for the order-preserving path).
__global__ void k_dict_compact(dtable t, uint64_t empty, int kw, void* out_keys, unsigned long long* counter,
                               int64_t* out_slots) {
    int64_t cap = (int64_t)t.mask + 1;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s <= cap; s += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long k = t.keys[s];
        bool live = s < cap ? k != empty : k == empty;
        if (!live) continue;
        unsigned long long p = atomicAdd(counter, 1ull);
        if (kw == 4) static_cast<unsigned*>(out_keys)[p] = (unsigned)k;
        else static_cast<unsigned long long*>(out_keys)[p] = k;
        out_slots[p] = s;
    }
}
__global__ void k_dict_rank(const int64_t* __restrict__ sorted_src, const int64_t* __restrict__ slots, int64_t m,
                            dtable t) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x)
        t.codes[slots[sorted_src[r]]] = (unsigned long long)r;
}

struct table_bufs {
    dbuf keys, codes, flags;
    dtable t;
};

table_bufs make_table(int64_t cap, int kw, cudaStream_t s) {
    table_bufs b;
    b.keys = dbuf((size_t)(cap + 1) * 8, s);
    b.codes = dbuf((size_t)(cap + 1) * 8, s);
    b.flags = dbuf(16, s);
    uint64_t empty = kw == 4 ? D_EMPTY4 : D_EMPTY8;
    fill_u64(b.keys.get(), empty, cap, s);
    fill_u64(b.keys.get<char>() + cap * 8, empty ^ 1ull, 1, s);  // sentinel slot starts unused
    fill_u64(b.codes.get(), NO_CODE, cap + 1, s);
    GX_CUDA(cudaMemsetAsync(b.flags.get(), 0, 16, s));
    b.t.keys = b.keys.get<unsigned long long>();
    b.t.codes = b.codes.get<unsigned long long>();
    b.t.mask = (uint64_t)cap - 1;
    b.t.overflow = b.flags.get<int>();
    return b;
}

col widen_if_narrow(const col& c, owned_col& hold, cudaStream_t s) {
    if (size_of(c.type) >= 4) return c;
    hold = widen_to_32(c, s);
    col w = c;
    w.data = hold.buf.get();
    w.type = hold.type;
    return w;
}

void check_encode(const col& c, int encode_type) {
    if (c.type == GX_STRING) fail(GX_EINVAL, "Cannot dictionary encode column of type STRING");
    require(is_numeric(c.type), "dictionary encode: unsupported column type " + type_name(c.type));
    if (!(is_signed_int(encode_type) || is_unsigned_int(encode_type)))
        fail(GX_EINVAL, "Encoded type must be integral, got " + type_name(encode_type));
}

int64_t table_capacity(const col& key, int64_t hint, double load_factor, cudaStream_t s) {
    int64_t est;
    if (hint > 0) est = hint;
    else if (key.n <= (1 << 16)) est = key.n;
    else est = std::min<int64_t>(key.n, ndv_estimate(key, s) * 9 / 8 + 64);
    double lf = load_factor > 0.05 && load_factor < 0.95 ? load_factor : 0.25;
    if (lf < 0.5 && est > (1 << 22)) lf = 0.5;  // keep very large tables compact
    return (int64_t)next_pow2((uint64_t)std::max<double>(64.0, std::ceil((double)est / lf)));
}

}  // namespace

// mode: 0 = hash codes, 1 = order-preserving codes.
void dictionary_encode(const gx_column_view& v, int encode_type, int64_t size_hint, double load_factor, int mode,
                       cudaStream_t s, gx_column* out, int64_t* dict_size) {
    col c0 = resolve(v);
    check_encode(c0, encode_type);
    owned_col hold;
    col c = widen_if_narrow(c0, hold, s);
    const int kw = size_of(c.type);
    const int kind = vkind_of(c.type);
    const int ow = size_of(encode_type);
    owned_col res = make_col(encode_type, c.n, s);
    int64_t cap = table_capacity(c, size_hint, load_factor, s);
    for (int attempt = 0; attempt < 6; ++attempt, cap *= 4) {
        table_bufs tb = make_table(cap, kw, s);
        unsigned long long* counter = reinterpret_cast<unsigned long long*>(tb.flags.get<char>() + 8);
        int g = grid_for(c.n, 256, 8);
        if (c.n > 0) {
            GX_PROF("dict_insert", s);
            if (kw == 4) k_dict_insert<4><<<g, 256, 0, s>>>(c.data, c.n, kind, tb.t, mode == 0, counter);
            else k_dict_insert<8><<<g, 256, 0, s>>>(c.data, c.n, kind, tb.t, mode == 0, counter);
            GX_LAUNCHED();
        }
        int hflags[4];
        GX_CUDA(cudaMemcpyAsync(hflags, tb.flags.get(), 16, cudaMemcpyDeviceToHost, s));
        GX_CUDA(cudaStreamSynchronize(s));
        if (hflags[0]) continue;
        unsigned long long ndv_u;
        std::memcpy(&ndv_u, &hflags[2], 8);
        int64_t ndv = (int64_t)ndv_u;
        if (mode == 1 && ndv > 0) {
            dbuf dk((size_t)ndv * kw, s), dslot((size_t)ndv * 8, s), cnt(8, s);
            GX_CUDA(cudaMemsetAsync(cnt.get(), 0, 8, s));
            uint64_t empty = kw == 4 ? D_EMPTY4 : D_EMPTY8;
            k_dict_compact<<<grid_for(cap + 1, 256, 8), 256, 0, s>>>(tb.t, empty, kw, dk.get(), cnt.get<unsigned long long>(),
                                                                   dslot.get<int64_t>());
            GX_LAUNCHED();
            // Sort distinct keys (with their compaction index) in value order.
            col kc;
            kc.data = dk.get();
            kc.n = ndv;
            kc.type = c.type;
            dbuf sk((size_t)ndv * kw, s), si((size_t)ndv * 8, s);
            radix_sort(kc, nullptr, 8, true, 0, -1, false, sk.get(), si.get(), nullptr, 0, s);
            k_dict_rank<<<grid_for(ndv, 256, 8), 256, 0, s>>>(si.get<int64_t>(), dslot.get<int64_t>(), ndv, tb.t);
            GX_LAUNCHED();
        }
        if (c.n > 0) {
            GX_PROF("dict_lookup", s);
            if (kw == 4) k_dict_lookup<4><<<g, 256, 0, s>>>(c.data, c.n, kind, tb.t, res.buf.get(), ow, 0);
            else k_dict_lookup<8><<<g, 256, 0, s>>>(c.data, c.n, kind, tb.t, res.buf.get(), ow, 0);
            GX_LAUNCHED();
        }
        GX_CUDA(cudaStreamSynchronize(s));
        *dict_size = ndv;
        *out = to_gx_column(std::move(res));
        return;
    }
    fail(GX_EOVERFLOW, "dictionary table overflow after retries");
}

void dictionary_encode_with_dict(const gx_column_view& v, const gx_column_view& dv, int encode_type, cudaStream_t s,
                                 gx_column* out) {
    col c0 = resolve(v), d0 = resolve(dv);
    if (encode_type != GX_INT32) fail(GX_EINVAL, "Unsupported encoded type");
    require(is_numeric(c0.type), "Dictionary encoding is not supported for non-integral type.");
    require(c0.type == d0.type, "dictionary encode: dictionary type differs from column type");
    owned_col h1, h2;
    col c = widen_if_narrow(c0, h1, s), d = widen_if_narrow(d0, h2, s);
    const int kw = size_of(c.type);
    const int kind = vkind_of(c.type);
    owned_col res = make_col(GX_INT32, c.n, s);
    // The reference sizes its map at dict.size() / 0.3 (dictionary_encode_dict_ready.cu:35-36).
    int64_t cap = (int64_t)next_pow2((uint64_t)std::max<double>(64.0, std::ceil(d.n / 0.3)));
    for (int attempt = 0; attempt < 6; ++attempt, cap *= 4) {
        table_bufs tb = make_table(cap, kw, s);
        if (d.n > 0) {
            int g = grid_for(d.n, 256, 8);
            if (kw == 4) k_dict_insert_positions<4><<<g, 256, 0, s>>>(d.data, d.n, kind, tb.t);
            else k_dict_insert_positions<8><<<g, 256, 0, s>>>(d.data, d.n, kind, tb.t);
            GX_LAUNCHED();
        }
        int ovf = read_scalar(tb.flags.get<int>(), s);
        if (ovf) continue;
        if (c.n > 0) {
            int g = grid_for(c.n, 256, 8);
            uint64_t missing = (uint64_t)(uint32_t)0x80000000u;
            if (kw == 4) k_dict_lookup<4><<<g, 256, 0, s>>>(c.data, c.n, kind, tb.t, res.buf.get(), 4, missing);
            else k_dict_lookup<8><<<g, 256, 0, s>>>(c.data, c.n, kind, tb.t, res.buf.get(), 4, missing);
            GX_LAUNCHED();
        }
        GX_CUDA(cudaStreamSynchronize(s));
        *out = to_gx_column(std::move(res));
        return;
    }
    fail(GX_EOVERFLOW, "dictionary table overflow after retries");
}

}  // namespace gx
