// gx_radix.cu — stable LSD radix sort / radix partition.
//
// Replaces the CUB DeviceRadixSort calls behind gamax::sort::{sort_column_pair,
// sort_column, argsort} (src/cuda/operators/sort/sort.cu:15-215) and the
// partition wrappers that delegate to them (src/cuda/operators/partition/
// partition.cu:11-99).  Semantics kept: stable, sorts on bits
// [begin_bit, end_bit) of the order-preserving key image (signed ints flip
// the sign bit, floats use the sign-magnitude twiddle with -0.0 == +0.0),
// descending order is stable too.
//
// Per 8-bit digit pass:
//   1. k_radix_hist  — one CTA per 4096-row tile, shared-memory histogram,
//                      counts written bin-major [bin][tile];
//   2. exclusive scan of the counts -> global start of (bin, tile);
//   3. scatter — where keys and values are 16-byte aligned 4/8-byte
//                      columns, the persistent bulk-copy scatter of the
//                      partition plan (radix_pass_bulk, key-image digits,
//                      stable ranking); otherwise k_radix_scatter: warp-level
//                      multisplit (match.any ranks rows with equal digits in
//                      input order), tile reordered by digit in shared
//                      memory, then written out in digit runs so each run is
//                      a contiguous, coalesced store.
#include <algorithm>

#include "gx_groupby.h"

namespace gx {
namespace {

constexpr int RS_NT = 512;
constexpr int RS_WARPS = RS_NT / 32;
constexpr int RS_IPT = 8;
constexpr int RS_TILE = RS_NT * RS_IPT;
constexpr int RS_MAXBITS = 8;
constexpr int RS_BINS = 1 << RS_MAXBITS;

template <int KW>
__device__ __forceinline__ uint64_t load_key(const void* p, int64_t i) {
    if (KW == 4) return __ldg(static_cast<const unsigned*>(p) + i);
    return __ldg(static_cast<const unsigned long long*>(p) + i);
}

template <int KW>
__global__ void __launch_bounds__(RS_NT) k_radix_hist(const void* __restrict__ keys, int64_t n, img_params ip,
                                                       int shift, int dbits, int64_t ntiles,
                                                       int64_t* __restrict__ counts) {
    __shared__ unsigned hist[RS_BINS];
    const int bins = 1 << dbits;
    for (int b = threadIdx.x; b < bins; b += RS_NT) hist[b] = 0;
    __syncthreads();
    int64_t base = blockIdx.x * (int64_t)RS_TILE;
#pragma unroll
    for (int k = 0; k < RS_IPT; ++k) {
        int64_t i = base + k * RS_NT + threadIdx.x;
        if (i < n) {
            uint64_t img = key_image<KW>(load_key<KW>(keys, i), ip);
            unsigned d = (unsigned)((img >> shift) & (uint64_t)(bins - 1));
            atomicAdd(&hist[d], 1u);
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < bins; b += RS_NT) counts[(int64_t)b * ntiles + blockIdx.x] = hist[b];
}

template <int KW, int VW, bool IOTA>
__global__ void __launch_bounds__(RS_NT) k_radix_scatter(const void* __restrict__ keys_in,
                                                          const void* __restrict__ vals_in, int64_t n,
                                                          img_params ip, int shift, int dbits,
                                                          int64_t ntiles,
                                                          const int64_t* __restrict__ offsets,
                                                          void* __restrict__ keys_out,
                                                          void* __restrict__ vals_out) {
    using kt = typename std::conditional<KW == 4, uint32_t, unsigned long long>::type;
    using vt = typename std::conditional<VW == 4, uint32_t, unsigned long long>::type;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned* whist = reinterpret_cast<unsigned*>(smem);                    // [WARPS][BINS]
    int64_t* gbase = reinterpret_cast<int64_t*>(smem + RS_WARPS * RS_BINS * 4);  // [BINS]
    unsigned* dbase = reinterpret_cast<unsigned*>(gbase + RS_BINS);          // [BINS + 1]
    kt* skeys = reinterpret_cast<kt*>(dbase + RS_BINS + 4);
    vt* svals = reinterpret_cast<vt*>(skeys + RS_TILE);

    const int bins = 1 << dbits;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < RS_WARPS * RS_BINS; i += RS_NT) whist[i] = 0;
    __syncthreads();

    const int64_t tile_base = blockIdx.x * (int64_t)RS_TILE;
    const int tile_n = (int)min((int64_t)RS_TILE, n - tile_base);
    const unsigned lt_mask = (1u << lane) - 1u;

    kt key[RS_IPT];
    vt val[RS_IPT];
    unsigned dig[RS_IPT];
    unsigned rank[RS_IPT];
#pragma unroll
    for (int k = 0; k < RS_IPT; ++k) {
        int local = warp * 32 * RS_IPT + k * 32 + lane;  // warp-striped: stable order (k, lane)
        int64_t i = tile_base + local;
        bool valid = local < tile_n;
        key[k] = valid ? (kt)load_key<KW>(keys_in, i) : (kt)0;
        if (VW) {
            if (IOTA) val[k] = (vt)i;
            else if (valid) val[k] = VW == 4 ? (vt)__ldg(static_cast<const unsigned*>(vals_in) + i)
                                             : (vt)__ldg(static_cast<const unsigned long long*>(vals_in) + i);
        }
        unsigned d = valid ? (unsigned)((key_image<KW>((uint64_t)key[k], ip) >> shift) & (uint64_t)(bins - 1))
                           : 0xFFFFu;
        dig[k] = d;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned r = __popc(peers & lt_mask);
        unsigned prior = valid ? whist[warp * RS_BINS + d] : 0;
        rank[k] = prior + r;
        __syncwarp();
        if (valid && r == 0) whist[warp * RS_BINS + d] = prior + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // Exclusive prefix over warps per digit, tile-local digit bases, global bases.
    if (threadIdx.x < RS_BINS) {
        unsigned run = 0;
        if (threadIdx.x < bins) {
            for (int w = 0; w < RS_WARPS; ++w) {
                unsigned c = whist[w * RS_BINS + threadIdx.x];
                whist[w * RS_BINS + threadIdx.x] = run;
                run += c;
            }
        }
        dbase[threadIdx.x] = run;  // digit total for now
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        // exclusive scan of RS_BINS digit totals by one warp (8 per lane)
        unsigned v[RS_BINS / 32];
        unsigned s = 0;
#pragma unroll
        for (int j = 0; j < RS_BINS / 32; ++j) {
            v[j] = dbase[lane * (RS_BINS / 32) + j];
            s += v[j];
        }
        unsigned inc = dev_::warp_inclusive_sum(s);
        unsigned run = inc - s;
#pragma unroll
        for (int j = 0; j < RS_BINS / 32; ++j) {
            dbase[lane * (RS_BINS / 32) + j] = run;
            run += v[j];
        }
    }
    __syncthreads();
    if (threadIdx.x < bins)
        gbase[threadIdx.x] = offsets[(int64_t)threadIdx.x * ntiles + blockIdx.x] - (int64_t)dbase[threadIdx.x];
#pragma unroll
    for (int k = 0; k < RS_IPT; ++k) {
        int local = warp * 32 * RS_IPT + k * 32 + lane;
        if (local < tile_n) {
            unsigned pos = dbase[dig[k]] + whist[warp * RS_BINS + dig[k]] + rank[k];
            skeys[pos] = key[k];
            if (VW) svals[pos] = val[k];
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < tile_n; j += RS_NT) {
        kt kk = skeys[j];
        unsigned d = (unsigned)((key_image<KW>((uint64_t)kk, ip) >> shift) & (uint64_t)(bins - 1));
        int64_t o = gbase[d] + j;
        static_cast<kt*>(keys_out)[o] = kk;
        if (VW) static_cast<vt*>(vals_out)[o] = svals[j];
    }
}

size_t scatter_smem(int kw, int vw) {
    return (size_t)RS_WARPS * RS_BINS * 4 + RS_BINS * 8 + (RS_BINS + 4) * 4 + (size_t)RS_TILE * (kw + vw);
}

// The scatter needs more than the default 48 KB of dynamic shared memory,
// so each instantiation's limit is raised once per device before its first
// launch.
template <int KW, int VW, bool IOTA>
void prepare_scatter() {
    static per_device_flag attr;
    attr.once([] {
        GX_CUDA(cudaFuncSetAttribute(k_radix_scatter<KW, VW, IOTA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)scatter_smem(KW, VW)));
    });
}

template <int KW, int VW, bool IOTA>
void launch_scatter(int64_t ntiles, cudaStream_t s, const void* kin, const void* vin, int64_t n,
                    const img_params& ip, int shift, int dbits, const int64_t* off, void* kout,
                    void* vout) {
    size_t smem = scatter_smem(KW, VW);
    prepare_scatter<KW, VW, IOTA>();
    k_radix_scatter<KW, VW, IOTA><<<(unsigned)ntiles, RS_NT, smem, s>>>(kin, vin, n, ip, shift, dbits,
                                                                       ntiles, off, kout, vout);
    GX_LAUNCHED();
}

void scatter_dispatch(int kw, int vw, bool iota, int64_t ntiles, cudaStream_t s, const void* kin,
                      const void* vin, int64_t n, const img_params& ip, int shift, int dbits,
                      const int64_t* off, void* kout, void* vout) {
#define GX_RS_CASE(K, V, I)                                                                   \
    if (kw == K && vw == V && iota == I) {                                                  \
        launch_scatter<K, V, I>(ntiles, s, kin, vin, n, ip, shift, dbits, off, kout, vout); \
        return;                                                                             \
    }
    GX_RS_CASE(4, 0, false)
    GX_RS_CASE(8, 0, false)
    GX_RS_CASE(4, 4, false)
    GX_RS_CASE(4, 8, false)
    GX_RS_CASE(8, 4, false)
    GX_RS_CASE(8, 8, false)
    GX_RS_CASE(4, 8, true)
    GX_RS_CASE(8, 8, true)
#undef GX_RS_CASE
    fail(GX_EUNSUPPORTED, "radix sort: unsupported key/value width combination");
}

template <int KW>
__global__ void k_image_range(const void* __restrict__ keys, int64_t n, img_params ip,
                              unsigned long long* __restrict__ out) {
    uint64_t lo = ~0ull, hi = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t img = key_image<KW>(load_key<KW>(keys, i), ip);
        lo = img < lo ? img : lo;
        hi = img > hi ? img : hi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(out, (unsigned long long)lo);
        atomicMax(out + 1, (unsigned long long)hi);
    }
}

template <typename S, typename D>
__global__ void k_narrow(D* __restrict__ out, const S* __restrict__ in, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (D)in[i];
}

}  // namespace

size_t radix_temp_bytes(int64_t n, int key_width, int val_width) {
    int kw = key_width < 4 ? 4 : key_width;
    int64_t ntiles = ceil_div(std::max<int64_t>(n, 1), RS_TILE);
    // Seven sub-buffers (the last an error flag), each rounded up to 256
    // bytes: 7 * 256 of slack.
    size_t b = (size_t)n * (kw + val_width);
    b += (size_t)RS_BINS * ntiles * 8 * 2 + 8;
    if (key_width < 4) b += (size_t)n * 4 * 2;
    return b + 7 * 256 + 256;
}

void key_image_range(const col& keys, uint64_t* lo, uint64_t* hi, cudaStream_t s) {
    int w = size_of(keys.type);
    require(w == 4 || w == 8, "key_image_range: 4/8-byte keys only");
    img_params ip{vkind_of(keys.type), w, 0, 0};
    dbuf out(16, s);
    uint64_t init[2] = {~0ull, 0ull};
    GX_CUDA(cudaMemcpyAsync(out.get(), init, 16, cudaMemcpyHostToDevice, s));
    if (keys.n > 0) {
        int g = grid_for(keys.n, 256, 8);
        if (w == 4) k_image_range<4><<<g, 256, 0, s>>>(keys.data, keys.n, ip, out.get<unsigned long long>());
        else k_image_range<8><<<g, 256, 0, s>>>(keys.data, keys.n, ip, out.get<unsigned long long>());
        GX_LAUNCHED();
    }
    uint64_t h[2];
    GX_CUDA(cudaMemcpyAsync(h, out.get(), 16, cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaStreamSynchronize(s));
    *lo = h[0];
    *hi = h[1];
}

// Internal entry with an optional image bias (sort on img - bias).
void radix_sort_biased(const col& keys_c, const void* vals_in, int val_width, bool vals_iota,
                       int begin_bit, int end_bit, bool descending, uint64_t bias, void* keys_out,
                       void* vals_out, void* temp, size_t temp_bytes, cudaStream_t s) {
    const int64_t n = keys_c.n;
    int lw = size_of(keys_c.type);
    require(lw > 0, "radix sort: non-numeric key type " + type_name(keys_c.type));
    require(val_width == 0 || val_width == 4 || val_width == 8 ||
                (val_width > 0 && vals_iota),
            "radix sort: value width must be 0, 4 or 8");
    if (vals_iota) val_width = 8;
    int full = 8 * lw;
    if (end_bit <= 0 || end_bit > full) end_bit = full;
    if (begin_bit < 0) begin_bit = 0;
    if (n == 0) return;

    dbuf own;
    char* tp = static_cast<char*>(temp);
    size_t need = radix_temp_bytes(n, lw, val_width);
    if (!tp || temp_bytes < need) {
        own = dbuf(need, s);
        tp = own.get<char>();
    }
    auto take = [&](size_t bytes) {
        char* p = tp;
        tp += (bytes + 255) & ~size_t(255);
        return p;
    };

    // Narrow keys: sort a 32-bit widened copy with the narrow image, then narrow back.
    col keys = keys_c;
    void* kout = keys_out;
    char* wide_out = nullptr;
    int kw = lw;
    if (lw < 4) {
        owned_col wc = widen_to_32(keys_c, s);
        char* wide_in = take((size_t)n * 4);
        GX_CUDA(cudaMemcpyAsync(wide_in, wc.buf.get(), (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
        keys.data = wide_in;
        wide_out = take((size_t)n * 4);
        kout = wide_out;
        kw = 4;
    }
    img_params ip{vkind_of(keys_c.type), lw, descending ? 1 : 0, bias};

    int nbits = end_bit - begin_bit;
    int passes = nbits > 0 ? (nbits + RS_MAXBITS - 1) / RS_MAXBITS : 0;
    if (passes == 0) {
        GX_CUDA(cudaMemcpyAsync(kout, keys.data, (size_t)n * kw, cudaMemcpyDeviceToDevice, s));
        if (val_width) {
            if (vals_iota) sequence_i64(static_cast<int64_t*>(vals_out), n, 0, 1, s);
            else GX_CUDA(cudaMemcpyAsync(vals_out, vals_in, (size_t)n * val_width, cudaMemcpyDeviceToDevice, s));
        }
    } else {
        int64_t ntiles = ceil_div(n, RS_TILE);
        char* tk = take((size_t)n * kw);
        char* tv = val_width ? take((size_t)n * val_width) : nullptr;
        int64_t* counts = reinterpret_cast<int64_t*>(take((size_t)RS_BINS * ntiles * 8));
        int64_t* offs = reinterpret_cast<int64_t*>(take((size_t)RS_BINS * ntiles * 8 + 8));
        int* err = reinterpret_cast<int*>(take(8));
        GX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
        bool bulk = false;
        const void* kin = keys.data;
        const void* vin = vals_in;
        bool iota = vals_iota;
        int shift = begin_bit;
        for (int p = 0; p < passes; ++p) {
            int dbits = std::min(RS_MAXBITS, end_bit - shift);
            bool to_out = ((passes - 1 - p) % 2) == 0;
            void* ko = to_out ? kout : tk;
            void* vo = to_out ? vals_out : tv;
            if (kw == 4) k_radix_hist<4><<<(unsigned)ntiles, RS_NT, 0, s>>>(kin, n, ip, shift, dbits, ntiles, counts);
            else k_radix_hist<8><<<(unsigned)ntiles, RS_NT, 0, s>>>(kin, n, ip, shift, dbits, ntiles, counts);
            GX_LAUNCHED();
            int64_t bins = 1 << dbits;
            exclusive_scan_i64(counts, offs, bins * ntiles, s);
            GX_PROF("radix_scatter", s);
            // Persistent bulk-copy pass where the columns allow it (16-byte
            // aligned 4/8-byte keys and values), else the per-tile kernel.
            if (radix_pass_bulk(kin, vin, kw, val_width, iota, n, ip, shift, dbits, RS_TILE, offs, ko, vo, err, s))
                bulk = true;
            else
                scatter_dispatch(kw, val_width, iota, ntiles, s, kin, vin, n, ip, shift, dbits, offs, ko, vo);
            kin = ko;
            vin = vo;
            iota = false;
            shift += dbits;
        }
        if (bulk && read_scalar(err, s)) fail(GX_ETIMEOUT, "radix sort: a bulk copy into shared memory did not complete");
    }
    if (lw < 4) {
        int g = grid_for(n, 256, 8);
        if (lw == 2) k_narrow<<<g, 256, 0, s>>>((uint16_t*)keys_out, (const uint32_t*)wide_out, n);
        else k_narrow<<<g, 256, 0, s>>>((uint8_t*)keys_out, (const uint32_t*)wide_out, n);
        GX_LAUNCHED();
    }
}

void radix_sort(const col& keys, const void* vals_in, int val_width, bool vals_iota, int begin_bit,
                int end_bit, bool descending, void* keys_out, void* vals_out, void* temp,
                size_t temp_bytes, cudaStream_t s) {
    radix_sort_biased(keys, vals_in, val_width, vals_iota, begin_bit, end_bit, descending, 0,
                      keys_out, vals_out, temp, temp_bytes, s);
}

}  // namespace gx

namespace gx {

// Scratch bytes radix_sort_pairs_scratch needs for n pairs of 4/8-byte keys
// and 4/8-byte values: both ping-pong halves, the per-tile digit counts and
// offsets, and the scan's temporaries (each rounded to 256 bytes).
size_t radix_pairs_scratch_bytes(int64_t n, int key_width, int val_width) {
    auto r256 = [](size_t b) { return (b + 255) & ~size_t(255); };
    int64_t ntiles = ceil_div(std::max<int64_t>(n, 1), RS_TILE);
    size_t b = r256((size_t)n * key_width) + r256((size_t)n * val_width);
    b += r256((size_t)RS_BINS * ntiles * 8) + r256((size_t)RS_BINS * ntiles * 8 + 8);
    return b + scan_scratch_bytes((int64_t)RS_BINS * ntiles);
}

// Raises the dynamic shared-memory limit of every 4/8-byte (key, value)
// scatter instantiation on the current device, so later pair sorts of any
// width combination launch without changing a kernel attribute.
void radix_prepare_pair_scatters() {
    prepare_scatter<4, 4, false>();
    prepare_scatter<4, 8, false>();
    prepare_scatter<8, 4, false>();
    prepare_scatter<8, 8, false>();
}

// The pass loop of radix_sort_biased (bias 0) for 4/8-byte keys and values,
// with every temporary taken from `scratch`.  The histogram and scatter
// kernels are the same, so the output equals gx_sort_column_pair's.  The
// caller has checked key/value widths and that scratch holds
// radix_pairs_scratch_bytes(n, kw, vw).  Nothing in scratch is read before
// it is written in the same call.
void radix_sort_pairs_scratch(const col& keys, const void* vals_in, int val_width, int begin_bit, int end_bit,
                              bool descending, void* keys_out, void* vals_out, char* scratch, cudaStream_t s) {
    const int64_t n = keys.n;
    const int kw = size_of(keys.type);
    int full = 8 * kw;
    if (end_bit <= 0 || end_bit > full) end_bit = full;
    if (begin_bit < 0) begin_bit = 0;
    if (n == 0) return;
    auto take = [&](size_t bytes) {
        char* p = scratch;
        scratch += (bytes + 255) & ~size_t(255);
        return p;
    };
    img_params ip{vkind_of(keys.type), kw, descending ? 1 : 0, 0};
    int nbits = end_bit - begin_bit;
    int passes = nbits > 0 ? (nbits + RS_MAXBITS - 1) / RS_MAXBITS : 0;
    if (passes == 0) {
        GX_CUDA(cudaMemcpyAsync(keys_out, keys.data, (size_t)n * kw, cudaMemcpyDeviceToDevice, s));
        GX_CUDA(cudaMemcpyAsync(vals_out, vals_in, (size_t)n * val_width, cudaMemcpyDeviceToDevice, s));
        return;
    }
    int64_t ntiles = ceil_div(n, RS_TILE);
    char* tk = take((size_t)n * kw);
    char* tv = take((size_t)n * val_width);
    int64_t* counts = reinterpret_cast<int64_t*>(take((size_t)RS_BINS * ntiles * 8));
    int64_t* offs = reinterpret_cast<int64_t*>(take((size_t)RS_BINS * ntiles * 8 + 8));
    char* scan_tmp = scratch;
    const void* kin = keys.data;
    const void* vin = vals_in;
    int shift = begin_bit;
    for (int p = 0; p < passes; ++p) {
        int dbits = std::min(RS_MAXBITS, end_bit - shift);
        bool to_out = ((passes - 1 - p) % 2) == 0;
        void* ko = to_out ? keys_out : tk;
        void* vo = to_out ? vals_out : tv;
        if (kw == 4) k_radix_hist<4><<<(unsigned)ntiles, RS_NT, 0, s>>>(kin, n, ip, shift, dbits, ntiles, counts);
        else k_radix_hist<8><<<(unsigned)ntiles, RS_NT, 0, s>>>(kin, n, ip, shift, dbits, ntiles, counts);
        GX_LAUNCHED();
        int64_t bins = 1 << dbits;
        exclusive_scan_i64_scratch(counts, offs, bins * ntiles, scan_tmp, s);
        scatter_dispatch(kw, val_width, false, ntiles, s, kin, vin, n, ip, shift, dbits, offs, ko, vo);
        kin = ko;
        vin = vo;
        shift += dbits;
    }
}

}  // namespace gx
