// gx_keys.cu — group keys that are not one numeric column.
//
// The reference groups STRING keys and multi-column keys with row hashers
// over every key column (src/cuda/memory/row_utils.cuh:61-95,
// operators/groupby/groupby_hash.cu:437-498), and with smart key fusion
// (hint.enable_skf) packs integral key columns into one 64-bit key
// (compress/multikey_compress.cu:25-399, operators/groupby/groupby.cu:403-465).
// Here every such request becomes a single integer key per row, so the one
// numeric group-by engine (HASH / SORT / PARTITION) runs unchanged:
//   * smart key fusion: each integral column contributes (value - min) on
//     ceil(log2(range + 1)) bits, or its dictionary code when the range saves
//     fewer than 2/3 of the column's bits; the packed key must fit 64 bits;
//   * otherwise (STRING, float or too-wide keys): each column is dictionary-
//     encoded (strings by content) and the codes are chained column by
//     column — code' = dense code of (code << 32 | next column's code) —
//     which is exact for any number of columns.
// The group-by then carries ANY(row id) and the original key columns of each
// group are gathered at that row (strings included), as the reference's SKF
// path does (groupby.cu:437-463).
#include <algorithm>

#include "gx_groupby.h"

namespace gx {
namespace {

int bits_for_range(uint64_t range) {
    int b = 0;
    while (b < 64 && (uint64_t(1) << b) <= range) ++b;
    return b;
}

constexpr int MAX_FUSE = 16;

struct fuse_desc {
    int n;
    const void* data[MAX_FUSE];
    int width[MAX_FUSE];   // bytes of the column read (dictionary codes: 8)
    int kind[MAX_FUSE];    // VK_I / VK_U
    uint64_t minv[MAX_FUSE];
    int shift[MAX_FUSE];
};

__device__ __forceinline__ uint64_t ld_int(const void* p, int w, int kind, int64_t i) {
    switch (w) {
        case 1: return kind == VK_I ? (uint64_t)(int64_t)static_cast<const int8_t*>(p)[i] : static_cast<const uint8_t*>(p)[i];
        case 2: return kind == VK_I ? (uint64_t)(int64_t)static_cast<const int16_t*>(p)[i] : static_cast<const uint16_t*>(p)[i];
        case 4: return kind == VK_I ? (uint64_t)(int64_t)static_cast<const int32_t*>(p)[i] : static_cast<const uint32_t*>(p)[i];
        default: return static_cast<const uint64_t*>(p)[i];
    }
}

__global__ void k_fuse(fuse_desc d, int64_t n, uint64_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = 0;
        for (int c = 0; c < d.n; ++c) k |= (ld_int(d.data[c], d.width[c], d.kind[c], i) - d.minv[c]) << d.shift[c];
        out[i] = k;
    }
}

// (acc << 32 | code) of two dense code columns (each code < 2^32, as a
// dense code is below the row count); codes are 4 or 8 bytes wide.
__global__ void k_chain(const void* __restrict__ acc, int acc_w, const void* __restrict__ code, int code_w,
                        int64_t n, uint64_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t a = acc_w == 4 ? (uint64_t)static_cast<const uint32_t*>(acc)[i] : static_cast<const uint64_t*>(acc)[i];
        const uint64_t c = code_w == 4 ? (uint64_t)static_cast<const uint32_t*>(code)[i]
                                       : static_cast<const uint64_t*>(code)[i];
        out[i] = (a << 32) | c;
    }
}

// Lengths of the gathered strings (one per output row).
__global__ void k_str_lens(const int64_t* __restrict__ off, const int64_t* __restrict__ idx, int64_t n,
                           int64_t* __restrict__ lens) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = idx[i];
        lens[i] = off[r + 1] - off[r];
    }
}

// One warp per output string: its bytes copied with coalesced lane strides.
__global__ void k_str_copy(const char* __restrict__ chars, const int64_t* __restrict__ off,
                           const int64_t* __restrict__ idx, int64_t n, const int64_t* __restrict__ out_off,
                           char* __restrict__ out_chars) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t i = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5); i < n; i += warps) {
        const int64_t r = idx[i];
        const int64_t src = off[r], len = off[r + 1] - src, dst = out_off[i];
        for (int64_t b = lane; b < len; b += 32) out_chars[dst + b] = chars[src + b];
    }
}

}  // namespace

// Wraps a pool buffer returned through a gx_column as an owned column.
static owned_col own(const gx_column& c, cudaStream_t s) {
    owned_col o;
    o.type = c.type;
    o.size = c.size;
    o.buf = dbuf::adopt(c.data, (size_t)c.capacity_bytes, s);
    return o;
}

bool multikey_compress(const gx_table_view* key, int max_bits, cudaStream_t s, owned_col* out, int* total_bits) {
    const int64_t nc = key->num_columns;
    if (nc < 1 || nc > MAX_FUSE) return false;
    const int64_t n = key->columns[0].size;
    for (int64_t c = 0; c < nc; ++c) {
        const int t = key->columns[c].type;
        if (!(is_signed_int(t) || is_unsigned_int(t))) return false;
    }
    fuse_desc d;
    std::memset(&d, 0, sizeof(d));
    std::vector<owned_col> codes;
    int bits = 0;
    for (int64_t c = 0; c < nc; ++c) {
        const gx_column_view& v = key->columns[c];
        col k = resolve(v);
        const int w = size_of(v.type);
        int cb = 0;
        uint64_t mn = 0;
        const void* src = k.data;
        int sw = w, skind = vkind_of(v.type);
        if (n > 0) {
            uint64_t lo, hi;
            compute_min_max(k, &lo, &hi, s);
            const uint64_t range = hi - lo;  // int64 / uint64 difference, exact mod 2^64
            cb = bits_for_range(range);
            mn = lo;
            // A range that saves fewer than 2/3 of the bits tries dictionary
            // codes instead (the reference's threshold).
            if (8 * w - cb < 8 * w * 2 / 3) {
                int64_t ndv = 0;
                gx_column cc;
                dictionary_encode(v, GX_INT64, 0, 0.5, 0, s, &cc, &ndv);
                codes.push_back(own(cc, s));
                const int db = bits_for_range((uint64_t)ndv);
                if (db < cb) {
                    cb = db;
                    mn = 0;
                    src = codes.back().buf.get();
                    sw = 8;
                    skind = VK_U;
                }
            }
        }
        d.data[c] = src;
        d.width[c] = sw;
        d.kind[c] = skind;
        d.minv[c] = mn;
        d.shift[c] = bits;
        bits += cb;
    }
    if (bits > max_bits) return false;
    d.n = (int)nc;
    owned_col o = make_col(GX_UINT64, n, s);
    if (n > 0) {
        k_fuse<<<grid_for(n, 256, 8), 256, 0, s>>>(d, n, o.buf.get<uint64_t>());
        GX_LAUNCHED();
    }
    GX_CUDA(cudaStreamSynchronize(s));
    *out = std::move(o);
    if (total_bits) *total_bits = bits;
    return true;
}

owned_col derive_group_key(const gx_table_view* key, bool skf, cudaStream_t s, int64_t* groups_bound) {
    const int64_t n = key->columns[0].size;
    owned_col fused;
    int bits = 0;
    if (skf && multikey_compress(key, 64, s, &fused, &bits)) {
        *groups_bound = bits >= 62 ? n : std::min<int64_t>(n, int64_t(1) << bits);
        return fused;
    }
    int64_t ndv = 0;
    gx_column c0;
    const gx_column_view& v0 = key->columns[0];
    if (v0.type == GX_STRING) dictionary_encode_strings(v0, 0, s, &c0, &ndv);
    else dictionary_encode(v0, GX_INT64, 0, 0.5, 0, s, &c0, &ndv);
    owned_col acc = own(c0, s);  // int32 codes for strings, int64 otherwise
    for (int64_t c = 1; c < key->num_columns; ++c) {
        int64_t nd = 0;
        gx_column cc;
        const gx_column_view& v = key->columns[c];
        if (v.type == GX_STRING) dictionary_encode_strings(v, 0, s, &cc, &nd);
        else dictionary_encode(v, GX_INT64, 0, 0.5, 0, s, &cc, &nd);
        owned_col code = own(cc, s);
        owned_col pair = make_col(GX_UINT64, n, s);
        if (n > 0) {
            k_chain<<<grid_for(n, 256, 8), 256, 0, s>>>(acc.buf.get(), size_of(acc.type), code.buf.get(),
                                                        size_of(code.type), n, pair.buf.get<uint64_t>());
            GX_LAUNCHED();
        }
        gx_column_view pv{pair.buf.get(), n, GX_UINT64, 0};
        gx_column nc;
        dictionary_encode(pv, GX_INT64, 0, 0.5, 0, s, &nc, &ndv);
        acc = own(nc, s);
    }
    *groups_bound = std::max<int64_t>(ndv, 1);
    return acc;
}

owned_col gather_column(const gx_column_view& v, const int64_t* idx, int64_t n, cudaStream_t s) {
    if (v.type != GX_STRING) {
        col c = resolve(v);
        owned_col o = make_col(v.type, n, s);
        gather_bytes(o.buf.get(), c.data, idx, n, size_of(v.type), s);
        return o;
    }
    require(v.offset >= 0 && v.size >= 0, "gather: negative string column size or offset");
    const gx_string_columns* sc = static_cast<const gx_string_columns*>(v.data);
    require(n == 0 || (sc && sc->chars && sc->offsets), "gather: null string column");
    const int64_t* off = n ? sc->offsets + v.offset : nullptr;
    dbuf lens((size_t)std::max<int64_t>(n, 1) * 8, s);
    dbuf out_off((size_t)(n + 1) * 8, s);
    int64_t total = 0;
    if (n > 0) {
        k_str_lens<<<grid_for(n, 256, 8), 256, 0, s>>>(off, idx, n, lens.get<int64_t>());
        GX_LAUNCHED();
        exclusive_scan_i64(lens.get<int64_t>(), out_off.get<int64_t>(), n, s);
        total = read_scalar(out_off.get<int64_t>() + n, s);
    }
    owned_col o = make_string_col(n, total, s);
    if (n > 0) {
        GX_CUDA(cudaMemcpyAsync(o.buf.get(), out_off.get(), (size_t)(n + 1) * 8, cudaMemcpyDeviceToDevice, s));
        k_str_copy<<<grid_for(n, 8, 8), 256, 0, s>>>(sc->chars, off, idx, n, out_off.get<int64_t>(),
                                                     const_cast<char*>(o.str->chars));
        GX_LAUNCHED();
    } else {
        GX_CUDA(cudaMemsetAsync(o.buf.get(), 0, 8, s));
    }
    return o;
}

}  // namespace gx
