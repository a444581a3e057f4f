// gx_gen.cu — seeded, counter-based synthetic data generators.
//
// Every value is a pure function of (seed, stream id, row index), so any row
// range can be regenerated independently on the GPU or on the CPU.  The
// random source is the SplitMix64 output function applied to a Weyl
// sequence (Steele, Lea, Flood: "Fast splittable pseudorandom number
// generators", OOPSLA 2014).  Key distributions follow the reference's
// generators (src/cuda/benchmarks/groupby/groupby_util.cuh:101-118 for the
// shuffled `i % G` keys, src/cuda/data_gen/generator.cuh:346-484 for Zipf by
// inverse CDF over P(rank r) ∝ 1/(r+1)^s), restated with this RNG.
#include <cmath>

#include "gx_core.cuh"

namespace gx {

__host__ __device__ __forceinline__ uint64_t sm64_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t rng_base(uint64_t seed, uint64_t sid) {
    return sm64_mix(seed ^ sm64_mix(sid + 0xD1B54A32D192ED03ull));
}
__host__ __device__ __forceinline__ uint64_t rng_at(uint64_t base, uint64_t i) {
    return sm64_mix(base + (i + 1) * 0x9E3779B97F4A7C15ull);
}
__host__ __device__ __forceinline__ uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}
// Bijection on [0, 2^k): add, odd multiply, xor-shift per round.
__host__ __device__ __forceinline__ uint64_t perm_bits(uint64_t x, int k, uint64_t key) {
    if (k == 0) return 0;
    uint64_t mask = k >= 64 ? ~0ull : ((1ull << k) - 1);
    int sh = k / 2 + 1;
    for (int r = 0; r < 4; ++r) {
        uint64_t rk = sm64_mix(key + r);
        x = (x + rk) & mask;
        x = (x * (rk | 1ull)) & mask;
        x ^= (sh < 64 ? (x >> sh) : 0);
    }
    return x;
}
// Bijection on [0, n) by cycle walking over the enclosing power of two.
__host__ __device__ __forceinline__ uint64_t perm_range(uint64_t i, uint64_t n, int k, uint64_t key) {
    uint64_t x = i;
    do { x = perm_bits(x, k, key); } while (x >= n);
    return x;
}

namespace {

__device__ __forceinline__ uint64_t draw_rank(const gx_gen_spec& sp, uint64_t base, uint64_t i, uint64_t n,
                                              int k, uint64_t G) {
    switch (sp.dist) {
        case GX_DIST_CYCLIC: return perm_range(i, n, k, sp.seed ^ 0xA5A5A5A5ull) % G;
        case GX_DIST_ZIPF: {
            double u = (double)(rng_at(base, i) >> 11) * 0x1.0p-53;
            int64_t lo = 0, hi = (int64_t)G;
            while (lo < hi) {
                int64_t mid = lo + (hi - lo) / 2;
                if (sp.zipf_cdf[mid] <= u) lo = mid + 1;
                else hi = mid;
            }
            return (uint64_t)(lo < (int64_t)G ? lo : (int64_t)G - 1);
        }
        case GX_DIST_SEQUENCE: return i;
        case GX_DIST_ZIPF_APPROX: {
            // Invert F(x) = ((x+1)^(1-s) - 1) / ((G+1)^(1-s) - 1) (ln form at s = 1),
            // the continuous counterpart of P(rank r) ∝ 1/(r+1)^s.
            double u = (double)(rng_at(base, i) >> 11) * 0x1.0p-53;
            double s = sp.zipf_s, x;
            if (fabs(s - 1.0) < 1e-6) x = exp(u * log((double)G + 1.0)) - 1.0;
            else {
                double a = 1.0 - s;
                x = pow(1.0 + u * (pow((double)G + 1.0, a) - 1.0), 1.0 / a) - 1.0;
            }
            uint64_t r = x > 0.0 ? (uint64_t)x : 0;
            return r < G ? r : G - 1;
        }
        default: return mulhi64(rng_at(base, i), G);
    }
}

__global__ void k_gen_keys(void* out, int width, int64_t n, gx_gen_spec sp, int k) {
    uint64_t base = rng_base(sp.seed, sp.stream_id);
    uint64_t G = sp.groups > 0 ? (uint64_t)sp.groups : 1;
    uint64_t miss_base = rng_base(sp.seed, sp.stream_id ^ 0x6D15ull);
    uint64_t miss_thr = sp.miss_frac > 0.0 ? (uint64_t)(sp.miss_frac * 0x1.0p53) : 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t r;
        uint64_t m = miss_thr ? rng_at(miss_base, (uint64_t)i) : 0;
        if (miss_thr && (m >> 11) < miss_thr) r = G + mulhi64(sm64_mix(m), G);
        else r = draw_rank(sp, base, (uint64_t)i, (uint64_t)n, k, G);
        if (width == 4) {
            uint32_t v = sp.scatter ? fmix32((uint32_t)r ^ 0x5bd1e995u) : (uint32_t)r;
            static_cast<uint32_t*>(out)[i] = v;
        } else {
            uint64_t v = sp.scatter ? fmix64(r ^ 0x5bd1e9955bd1e995ull) : r;
            static_cast<uint64_t*>(out)[i] = v;
        }
    }
}

__global__ void k_gen_values(void* out, int type, int64_t n, gx_gen_spec sp) {
    uint64_t base = rng_base(sp.seed, sp.stream_id);
    uint64_t span = (uint64_t)(sp.hi - sp.lo);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t r = rng_at(base, (uint64_t)i);
        switch (type) {
            case GX_FLOAT64: static_cast<double*>(out)[i] = (double)(r >> 11) * 0x1.0p-53; break;
            case GX_FLOAT32: static_cast<float*>(out)[i] = (float)(r >> 40) * 0x1.0p-24f; break;
            case GX_INT64: case GX_UINT64:
                static_cast<int64_t*>(out)[i] = sp.lo + (int64_t)mulhi64(r, span);
                break;
            case GX_INT32: case GX_UINT32:
                static_cast<int32_t*>(out)[i] = (int32_t)(sp.lo + (int64_t)mulhi64(r, span));
                break;
            case GX_INT16: case GX_UINT16:
                static_cast<int16_t*>(out)[i] = (int16_t)(sp.lo + (int64_t)mulhi64(r, span));
                break;
            default:
                static_cast<int8_t*>(out)[i] = (int8_t)(sp.lo + (int64_t)mulhi64(r, span));
                break;
        }
    }
}

__global__ void k_gen_perm(void* out, int width, int64_t n, int k, uint64_t seed, int64_t base_v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t v = (int64_t)perm_range((uint64_t)i, (uint64_t)n, k, seed) + base_v;
        if (width == 4) static_cast<int32_t*>(out)[i] = (int32_t)v;
        else static_cast<int64_t*>(out)[i] = v;
    }
}

}  // namespace

void zipf_cdf_host(int64_t G, double s, double* cdf) {
    double total = 0.0;
    for (int64_t r = 0; r < G; ++r) {
        total += 1.0 / std::pow((double)(r + 1), s);
        cdf[r] = total;
    }
    for (int64_t r = 0; r < G; ++r) cdf[r] /= total;
    if (G > 0) cdf[G - 1] = 1.0;
}

void generate_keys(const gx_column_view& v, const gx_gen_spec& sp, cudaStream_t s) {
    col c = resolve(v);
    int w = size_of(c.type);
    require(w == 4 || w == 8, "generate_keys: 4- or 8-byte key column required");
    require(sp.dist != GX_DIST_ZIPF || sp.zipf_cdf != nullptr, "generate_keys: Zipf needs a CDF");
    if (c.n == 0) return;
    int k = ilog2_ceil((uint64_t)c.n);
    k_gen_keys<<<grid_for(c.n, 256, 8), 256, 0, s>>>(const_cast<void*>(c.data), w, c.n, sp, k);
    GX_LAUNCHED();
}

void generate_values(const gx_column_view& v, const gx_gen_spec& sp, cudaStream_t s) {
    col c = resolve(v);
    require(is_numeric(c.type), "generate_values: numeric column required");
    if (!is_float(c.type)) require(sp.hi > sp.lo, "generate_values: empty range");
    if (c.n == 0) return;
    k_gen_values<<<grid_for(c.n, 256, 8), 256, 0, s>>>(const_cast<void*>(c.data), c.type, c.n, sp);
    GX_LAUNCHED();
}

void generate_permutation(const gx_column_view& v, uint64_t seed, int64_t base_v, cudaStream_t s) {
    col c = resolve(v);
    int w = size_of(c.type);
    require(w == 4 || w == 8, "generate_permutation: 4- or 8-byte column required");
    if (c.n == 0) return;
    int k = ilog2_ceil((uint64_t)c.n);
    k_gen_perm<<<grid_for(c.n, 256, 8), 256, 0, s>>>(const_cast<void*>(c.data), w, c.n, k, seed, base_v);
    GX_LAUNCHED();
}

}  // namespace gx

namespace gx {
namespace {
__global__ void k_gen_strings(const char* __restrict__ dchars, const int64_t* __restrict__ doff, int64_t dsize,
                              const int32_t* __restrict__ codes, int64_t rows, const int64_t* __restrict__ off,
                              char* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t c = codes[i];
        if (c < 0 || c >= dsize) continue;
        const int64_t s = doff[c], len = doff[c + 1] - s;
        const int64_t o = off[i];
        if (off[i + 1] - o != len) continue;  // offsets must match the dictionary lengths
        for (int64_t j = 0; j < len; ++j) out[o + j] = dchars[s + j];
    }
}
}  // namespace

void generate_strings(const char* dchars, const int64_t* doff, int64_t dsize, const int32_t* codes, int64_t rows,
                      const int64_t* off, char* out, cudaStream_t s) {
    require(dchars && doff && codes && off && out, "generate_strings: null pointer");
    if (rows <= 0) return;
    k_gen_strings<<<grid_for(rows, 256, 8), 256, 0, s>>>(dchars, doff, dsize, codes, rows, off, out);
    GX_LAUNCHED();
}
}  // namespace gx
