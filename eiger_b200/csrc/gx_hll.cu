// gx_hll.cu — HyperLogLog distinct-count sketch and column statistics.
//
// Replaces gamax::stats::compute_ndv_approx (src/cuda/stats/stats_compute.cu:
// 103-196), which drives the plain AUTO strategy rule
// (src/cuda/operators/groupby/groupby.cu:68-119).  The reference uses
// cuCollections' hyperloglog with standard deviation 0.0122197, i.e. 2^13
// registers; this sketch uses the same register count.  Algorithm:
// Flajolet, Fusy, Gandouet, Meunier, "HyperLogLog: the analysis of a
// near-optimal cardinality estimation algorithm" (AofA 2007) with the
// linear-counting small-range correction; the 64-bit hash (MurmurHash3
// fmix64 of the canonical key bits) makes the large-range correction
// unnecessary.  Each CTA keeps its registers in shared memory and merges
// them into the global sketch with one atomicMax per non-zero register.
#include <cmath>

#include "gx_groupby.h"

namespace gx {

constexpr int HLL_P = 13;
constexpr int HLL_M = 1 << HLL_P;

__host__ __device__ __forceinline__ uint64_t hll_hash(uint64_t canon_bits) {
    return fmix64(canon_bits ^ 0x5bd1e9955bd1e995ull);
}
__host__ __device__ __forceinline__ void hll_index_rank(uint64_t h, uint32_t* idx, uint32_t* rank) {
    *idx = (uint32_t)(h >> (64 - HLL_P));
    uint64_t w = (h << HLL_P) | (1ull << (HLL_P - 1));  // guard bit bounds the rank
#ifdef __CUDA_ARCH__
    *rank = (uint32_t)__clzll((long long)w) + 1;
#else
    *rank = (uint32_t)__builtin_clzll(w) + 1;
#endif
}

namespace {

template <int KW>
__global__ void k_hll(const void* __restrict__ keys, int64_t n, int64_t stride, int kind,
                      unsigned* __restrict__ regs) {
    __shared__ unsigned sreg[HLL_M];
    for (int i = threadIdx.x; i < HLL_M; i += blockDim.x) sreg[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t b;
        if (KW == 4) b = canon32(__ldg(static_cast<const unsigned*>(keys) + i * stride), kind);
        else b = canon64(__ldg(static_cast<const unsigned long long*>(keys) + i * stride), kind);
        uint32_t idx, rank;
        hll_index_rank(hll_hash(b), &idx, &rank);
        if (sreg[idx] < rank) atomicMax(&sreg[idx], rank);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < HLL_M; i += blockDim.x)
        if (sreg[i]) atomicMax(&regs[i], sreg[i]);
}

// Full-column sketch of a 16-byte aligned key column: 16-byte loads, four
// in flight per thread (the strided kernel above keeps one 4-byte load in
// flight per thread, too few to cover HBM latency); the n % (16 / KW) tail
// keys are added by block 0.  Same registers as k_hll (max is order-free).
constexpr int HLLV_NT = 512, HLLV_VEC = 4;
template <int KW>
__global__ void __launch_bounds__(HLLV_NT) k_hll_vec(const void* __restrict__ keys, int64_t n, int kind,
                                                     unsigned* __restrict__ regs) {
    __shared__ unsigned sreg[HLL_M];
    for (int i = threadIdx.x; i < HLL_M; i += HLLV_NT) sreg[i] = 0;
    __syncthreads();
    auto add = [&](uint64_t b) {
        uint32_t idx, rank;
        hll_index_rank(hll_hash(b), &idx, &rank);
        if (sreg[idx] < rank) atomicMax(&sreg[idx], rank);
    };
    constexpr int KPV = 16 / KW;  // keys per 16-byte vector
    const int64_t nvec = n / KPV;
    const uint4* kv = static_cast<const uint4*>(keys);
    const int64_t step = (int64_t)gridDim.x * HLLV_NT;
    for (int64_t v0 = blockIdx.x * (int64_t)HLLV_NT + threadIdx.x; v0 < nvec; v0 += step * HLLV_VEC) {
        uint4 x[HLLV_VEC] = {};
#pragma unroll
        for (int q = 0; q < HLLV_VEC; ++q)
            if (v0 + q * step < nvec) x[q] = __ldcs(kv + v0 + q * step);
#pragma unroll
        for (int q = 0; q < HLLV_VEC; ++q) {
            if (v0 + q * step >= nvec) break;
            if (KW == 4) {
                add(canon32(x[q].x, kind));
                add(canon32(x[q].y, kind));
                add(canon32(x[q].z, kind));
                add(canon32(x[q].w, kind));
            } else {
                add(canon64(((uint64_t)x[q].y << 32) | x[q].x, kind));
                add(canon64(((uint64_t)x[q].w << 32) | x[q].z, kind));
            }
        }
    }
    if (blockIdx.x == 0)
        for (int64_t i = nvec * KPV + threadIdx.x; i < n; i += HLLV_NT) {
            if (KW == 4) add(canon32(__ldg(static_cast<const unsigned*>(keys) + i), kind));
            else add(canon64(__ldg(static_cast<const unsigned long long*>(keys) + i), kind));
        }
    __syncthreads();
    for (int i = threadIdx.x; i < HLL_M; i += HLLV_NT)
        if (sreg[i]) atomicMax(&regs[i], sreg[i]);
}

template <int KW>
__global__ void k_minmax(const void* __restrict__ keys, int64_t n, int kind, unsigned long long* out) {
    // Track the order-preserving image; convert back on the host.
    uint64_t lo = ~0ull, hi = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t img;
        if (KW == 4) img = ordered32(__ldg(static_cast<const unsigned*>(keys) + i), kind);
        else img = ordered64(__ldg(static_cast<const unsigned long long*>(keys) + i), kind);
        lo = img < lo ? img : lo;
        hi = img > hi ? img : hi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t a = __shfl_xor_sync(0xffffffffu, lo, o), b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(out, (unsigned long long)lo);
        atomicMax(out + 1, (unsigned long long)hi);
    }
}

}  // namespace

double hll_estimate(const unsigned* regs) {
    double m = HLL_M;
    double alpha = 0.7213 / (1.0 + 1.079 / m);
    double sum = 0.0;
    int zeros = 0;
    for (int i = 0; i < HLL_M; ++i) {
        sum += std::ldexp(1.0, -(int)regs[i]);
        zeros += regs[i] == 0;
    }
    double e = alpha * m * m / sum;
    if (e <= 2.5 * m && zeros > 0) e = m * std::log(m / (double)zeros);
    return e;
}

// Registers of the sketch over rows 0, stride, 2*stride, ... (n rows taken).
void hll_registers(const col& key_in, int64_t n, int64_t stride, unsigned* d_regs, cudaStream_t s) {
    owned_col widened;
    col key = key_in;
    if (size_of(key.type) < 4) {
        widened = widen_to_32(key, s);
        key.data = widened.buf.get();
        key.type = widened.type;
    }
    GX_CUDA(cudaMemsetAsync(d_regs, 0, HLL_M * sizeof(unsigned), s));
    if (n <= 0) return;
    int kind = vkind_of(key.type);
    const int kw = size_of(key.type);
    if (stride == 1 && reinterpret_cast<uintptr_t>(key.data) % 16 == 0 && n >= (int64_t)HLLV_NT * 16) {
        // Two CTAs per SM; fewer for small columns (each CTA merges 2^13
        // registers into the global sketch).
        const int g = (int)std::min<int64_t>((int64_t)dev().sm_count * 2, ceil_div(n, (int64_t)HLLV_NT * 64));
        if (kw == 4) k_hll_vec<4><<<g, HLLV_NT, 0, s>>>(key.data, n, kind, d_regs);
        else k_hll_vec<8><<<g, HLLV_NT, 0, s>>>(key.data, n, kind, d_regs);
        GX_LAUNCHED();
        return;
    }
    int g = grid_for(n, 256, 2);
    if (kw == 4) k_hll<4><<<g, 256, 0, s>>>(key.data, n, stride, kind, d_regs);
    else k_hll<8><<<g, 256, 0, s>>>(key.data, n, stride, kind, d_regs);
    GX_LAUNCHED();
}

int64_t ndv_estimate(const col& key, cudaStream_t s) {
    if (key.n == 0) return 0;
    dbuf regs(HLL_M * sizeof(unsigned), s);
    hll_registers(key, key.n, 1, regs.get<unsigned>(), s);
    std::vector<unsigned> h(HLL_M);
    GX_CUDA(cudaMemcpyAsync(h.data(), regs.get(), HLL_M * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaStreamSynchronize(s));
    return (int64_t)std::llround(hll_estimate(h.data()));
}

void compute_min_max(const col& key, void* min_out, void* max_out, cudaStream_t s) {
    int w = size_of(key.type);
    require(w > 0, "min/max of a non-numeric column");
    require(key.n > 0, "min/max of an empty column");
    owned_col widened;
    col k = key;
    if (w < 4) {
        widened = widen_to_32(key, s);
        k.data = widened.buf.get();
        k.type = widened.type;
    }
    dbuf out(16, s);
    uint64_t init[2] = {~0ull, 0ull};
    GX_CUDA(cudaMemcpyAsync(out.get(), init, 16, cudaMemcpyHostToDevice, s));
    int kind = vkind_of(k.type);
    int g = grid_for(k.n, 256, 8);
    if (size_of(k.type) == 4) k_minmax<4><<<g, 256, 0, s>>>(k.data, k.n, kind, out.get<unsigned long long>());
    else k_minmax<8><<<g, 256, 0, s>>>(k.data, k.n, kind, out.get<unsigned long long>());
    GX_LAUNCHED();
    uint64_t h[2];
    GX_CUDA(cudaMemcpyAsync(h, out.get(), 16, cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaStreamSynchronize(s));
    // Invert the order-preserving image, widen to int64 / uint64 / double.
    for (int j = 0; j < 2; ++j) {
        uint64_t img = h[j], raw;
        int kd = vkind_of(key.type);
        if (size_of(k.type) == 4) {
            uint32_t b = (uint32_t)img;
            if (kd == VK_I) raw = (uint64_t)(int64_t)(int32_t)(b ^ 0x80000000u);
            else if (kd == VK_F) {
                uint32_t f = (b & 0x80000000u) ? (b ^ 0x80000000u) : ~b;
                float fv;
                std::memcpy(&fv, &f, 4);
                double dv = fv;
                std::memcpy(&raw, &dv, 8);
            } else raw = b;
        } else {
            if (kd == VK_I) raw = img ^ 0x8000000000000000ull;
            else if (kd == VK_F) raw = (img & 0x8000000000000000ull) ? (img ^ 0x8000000000000000ull) : ~img;
            else raw = img;
        }
        std::memcpy(j == 0 ? min_out : max_out, &raw, 8);
    }
}

}  // namespace gx
