// gx_util.cu — allocator, device info and small device primitives shared by
// the operators (fill, scan, sequence, gather, widening).
#include <mutex>

#include "gx_core.cuh"

namespace gx {

std::atomic<int64_t> g_launches{0};
std::atomic<int> g_profiling{0};

namespace {
struct prof_rec {
    std::string name;
    cudaEvent_t a, b;
};
std::mutex g_prof_mu;
std::vector<prof_rec> g_prof;
}  // namespace

prof_scope::prof_scope(const char* n, cudaStream_t st) : name(n), s(st) {
    if (!g_profiling.load()) return;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
}
prof_scope::~prof_scope() {
    if (!a) return;
    cudaEventRecord(b, s);
    std::lock_guard<std::mutex> g(g_prof_mu);
    g_prof.push_back({name, a, b});
}

// Sum of recorded durations (ms) and counts for `name`; clears on reset.
void prof_read(const char* name, double* total_ms, int64_t* count, bool reset) {
    std::lock_guard<std::mutex> g(g_prof_mu);
    double t = 0;
    int64_t c = 0;
    for (auto& r : g_prof) {
        if (r.name != name) continue;
        cudaEventSynchronize(r.b);
        float ms = 0;
        cudaEventElapsedTime(&ms, r.a, r.b);
        t += ms;
        ++c;
    }
    if (total_ms) *total_ms = t;
    if (count) *count = c;
    if (reset) {
        for (auto& r : g_prof) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        g_prof.clear();
    }
}

namespace {
std::mutex g_dev_mu;
device_info g_dev[GX_MAX_DEVICES];
bool g_dev_ok[GX_MAX_DEVICES] = {};

std::atomic<int64_t> g_cur{0}, g_peak{0};
std::mutex g_size_mu;
// Allocation sizes for the stats; the pool itself is CUDA's.
struct size_rec { void* p; size_t n; };
std::vector<size_rec> g_sizes;
per_device_flag g_pool_ready;
}  // namespace

const device_info& dev() {
    int d = 0;
    GX_CUDA(cudaGetDevice(&d));
    if (d < 0 || d >= GX_MAX_DEVICES)
        fail(GX_EUNSUPPORTED, "device ordinal " + std::to_string(d) + " is beyond the " +
                                  std::to_string(GX_MAX_DEVICES) + " devices this library supports");
    std::lock_guard<std::mutex> g(g_dev_mu);
    if (!g_dev_ok[d]) {
        device_info i;
        i.device = d;
        GX_CUDA(cudaDeviceGetAttribute(&i.sm_count, cudaDevAttrMultiProcessorCount, d));
        GX_CUDA(cudaDeviceGetAttribute(&i.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d));
        GX_CUDA(cudaDeviceGetAttribute(&i.l2_bytes, cudaDevAttrL2CacheSize, d));
        g_dev[d] = i;
        g_dev_ok[d] = true;
    }
    return g_dev[d];
}

void* pool_alloc(size_t bytes, cudaStream_t s) {
    g_pool_ready.once([] {
        cudaMemPool_t pool;
        GX_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev().device));
        uint64_t thr = UINT64_MAX;
        GX_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    });
    // 256-byte granularity like the reference's slab (mem_manager.cu:102-128).
    size_t rounded = (bytes + 255) & ~size_t(255);
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, rounded, s);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(GX_ENOMEM, "device pool exhausted allocating " + std::to_string(bytes) + " bytes");
    }
    GX_CUDA(e);
    {
        std::lock_guard<std::mutex> g(g_size_mu);
        g_sizes.push_back({p, rounded});
    }
    int64_t cur = g_cur.fetch_add((int64_t)rounded) + (int64_t)rounded;
    int64_t pk = g_peak.load();
    while (cur > pk && !g_peak.compare_exchange_weak(pk, cur)) {}
    return p;
}

namespace {
struct scratch_set {
    struct buf {
        void* p = nullptr;
        size_t bytes = 0;
        int device = -1;
    };
    buf b[GX_MAX_DEVICES][SCRATCH_SLOTS];
    ~scratch_set() {
        for (auto& d : b)
            for (auto& x : d)
                if (x.p) {
                    cudaSetDevice(x.device);
                    cudaFree(x.p);  // errors ignored: the context may already be gone at exit
                }
    }
};
thread_local scratch_set t_scratch;
}  // namespace

void* thread_scratch(int slot, size_t bytes) {
    require(slot >= 0 && slot < SCRATCH_SLOTS, "scratch slot out of range");
    const int d = dev().device;
    auto& x = t_scratch.b[d][slot];
    if (x.bytes < bytes) {
        if (x.p) GX_CUDA(cudaFree(x.p));
        x.p = nullptr;
        x.bytes = 0;
        const size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&x.p, want);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            fail(GX_ENOMEM, "device memory exhausted allocating " + std::to_string(bytes) + " bytes of scratch");
        }
        GX_CUDA(e);
        x.bytes = want;
        x.device = d;
    }
    return x.p;
}

void pool_free(void* p, cudaStream_t s) {
    if (!p) return;
    size_t n = 0;
    {
        std::lock_guard<std::mutex> g(g_size_mu);
        for (size_t i = g_sizes.size(); i-- > 0;) {
            if (g_sizes[i].p == p) {
                n = g_sizes[i].n;
                g_sizes[i] = g_sizes.back();
                g_sizes.pop_back();
                break;
            }
        }
    }
    g_cur.fetch_sub((int64_t)n);
    cudaFreeAsync(p, s);
}

void pool_stats(int64_t* cur, int64_t* peak) {
    if (cur) *cur = g_cur.load();
    if (peak) *peak = g_peak.load();
}
void pool_reset_peak() { g_peak.store(g_cur.load()); }

std::string type_name(int t) {
    static const char* names[] = {"EMPTY", "INT8", "INT16", "INT32", "INT64", "BOOL8", "UINT8",
                                  "UINT16", "UINT32", "UINT64", "FLOAT32", "FLOAT64", "STRING"};
    return (t >= 0 && t < GX_NUM_TYPE_IDS) ? names[t] : "INVALID";
}

// ---------------------------------------------------------------------------
// Kernels.
// ---------------------------------------------------------------------------
namespace {

__global__ void k_fill_u64(uint64_t* __restrict__ d, uint64_t v, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) d[i] = v;
}
__global__ void k_fill_u32(uint32_t* __restrict__ d, uint32_t v, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) d[i] = v;
}
__global__ void k_sequence(int64_t* __restrict__ d, int64_t n, int64_t start, int64_t step) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) d[i] = start + i * step;
}

template <typename T>
__global__ void k_gather(T* __restrict__ out, const T* __restrict__ src,
                         const int64_t* __restrict__ idx, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) out[i] = src[idx[i]];
}

template <typename S, typename D>
__global__ void k_widen(D* __restrict__ out, const S* __restrict__ in, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) out[i] = (D)in[i];
}

constexpr int SCAN_NT = 512;
constexpr int SCAN_IPT = 8;
constexpr int SCAN_TILE = SCAN_NT * SCAN_IPT;

// Per-tile sums of int64 counts.
__global__ void __launch_bounds__(SCAN_NT) k_tile_sums(const int64_t* __restrict__ in, int64_t n,
                                                        int64_t* __restrict__ sums) {
    __shared__ int64_t sm[SCAN_NT / 32 + 1];
    int64_t base = blockIdx.x * (int64_t)SCAN_TILE;
    int64_t acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
        int64_t i = base + k * SCAN_NT + threadIdx.x;
        if (i < n) acc += in[i];
    }
    acc = dev_::warp_sum(acc);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        int64_t v = threadIdx.x < SCAN_NT / 32 ? sm[threadIdx.x] : 0;
        v = dev_::warp_sum(v);
        if (threadIdx.x == 0) sums[blockIdx.x] = v;
    }
}

// Exclusive scan of each tile seeded with the tile's prefix.
__global__ void __launch_bounds__(SCAN_NT) k_tile_scan(const int64_t* __restrict__ in, int64_t n,
                                                        const int64_t* __restrict__ tile_prefix,
                                                        int64_t* __restrict__ out) {
    __shared__ int64_t sm[SCAN_NT / 32 + 1];
    int64_t base = blockIdx.x * (int64_t)SCAN_TILE + threadIdx.x * (int64_t)SCAN_IPT;
    int64_t v[SCAN_IPT];
    int64_t local = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
        int64_t i = base + k;
        v[k] = i < n ? in[i] : 0;
        local += v[k];
    }
    int64_t total;
    int64_t excl = dev_::block_exclusive_sum<SCAN_NT>(local, sm, &total);
    int64_t run = tile_prefix[blockIdx.x] + excl;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
        int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

__global__ void k_set_last(const int64_t* __restrict__ tile_prefix, int64_t ntiles,
                           const int64_t* __restrict__ tile_sums, int64_t* __restrict__ out,
                           int64_t n) {
    if (threadIdx.x == 0 && blockIdx.x == 0)
        out[n] = ntiles ? tile_prefix[ntiles - 1] + tile_sums[ntiles - 1] : 0;
}

}  // namespace

void fill_u64(void* dst, uint64_t pattern, int64_t words, cudaStream_t s) {
    if (words <= 0) return;
    k_fill_u64<<<grid_for(words, 256, 8), 256, 0, s>>>(static_cast<uint64_t*>(dst), pattern, words);
    GX_LAUNCHED();
}
void fill_u32(void* dst, uint32_t pattern, int64_t words, cudaStream_t s) {
    if (words <= 0) return;
    k_fill_u32<<<grid_for(words, 256, 8), 256, 0, s>>>(static_cast<uint32_t*>(dst), pattern, words);
    GX_LAUNCHED();
}
void sequence_i64(int64_t* out, int64_t n, int64_t start, int64_t step, cudaStream_t s) {
    if (n <= 0) return;
    k_sequence<<<grid_for(n, 256, 8), 256, 0, s>>>(out, n, start, step);
    GX_LAUNCHED();
}

void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
    if (n <= 0) {
        fill_u64(out, 0, 1, s);
        return;
    }
    int64_t ntiles = ceil_div(n, SCAN_TILE);
    dbuf sums(ntiles * sizeof(int64_t), s), pref((ntiles + 1) * sizeof(int64_t), s);
    k_tile_sums<<<(unsigned)ntiles, SCAN_NT, 0, s>>>(in, n, sums.get<int64_t>());
    GX_LAUNCHED();
    if (ntiles == 1) {
        fill_u64(pref.get(), 0, 1, s);
    } else {
        exclusive_scan_i64(sums.get<int64_t>(), pref.get<int64_t>(), ntiles, s);
    }
    k_tile_scan<<<(unsigned)ntiles, SCAN_NT, 0, s>>>(in, n, pref.get<int64_t>(), out);
    GX_LAUNCHED();
    k_set_last<<<1, 32, 0, s>>>(pref.get<int64_t>(), ntiles, sums.get<int64_t>(), out, n);
    GX_LAUNCHED();
}

void gather_bytes(void* out, const void* src, const int64_t* idx, int64_t n, int width,
                  cudaStream_t s) {
    if (n <= 0) return;
    int g = grid_for(n, 256, 8);
    switch (width) {
        case 1: k_gather<<<g, 256, 0, s>>>((uint8_t*)out, (const uint8_t*)src, idx, n); break;
        case 2: k_gather<<<g, 256, 0, s>>>((uint16_t*)out, (const uint16_t*)src, idx, n); break;
        case 4: k_gather<<<g, 256, 0, s>>>((uint32_t*)out, (const uint32_t*)src, idx, n); break;
        case 8: k_gather<<<g, 256, 0, s>>>((uint64_t*)out, (const uint64_t*)src, idx, n); break;
        default: fail(GX_EINVAL, "gather: bad element width");
    }
    GX_LAUNCHED();
}

owned_col widen_to_32(const col& c, cudaStream_t s) {
    bool sgn = is_signed_int(c.type);
    owned_col o = make_col(sgn ? GX_INT32 : GX_UINT32, c.n, s);
    if (c.n == 0) return o;
    int g = grid_for(c.n, 256, 8);
    switch (c.type) {
        case GX_INT8: k_widen<<<g, 256, 0, s>>>(o.buf.get<int32_t>(), c.as<int8_t>(), c.n); break;
        case GX_INT16: k_widen<<<g, 256, 0, s>>>(o.buf.get<int32_t>(), c.as<int16_t>(), c.n); break;
        case GX_UINT8:
        case GX_BOOL8: k_widen<<<g, 256, 0, s>>>(o.buf.get<uint32_t>(), c.as<uint8_t>(), c.n); break;
        case GX_UINT16: k_widen<<<g, 256, 0, s>>>(o.buf.get<uint32_t>(), c.as<uint16_t>(), c.n); break;
        default: fail(GX_EINVAL, "widen_to_32: not a narrow integer type");
    }
    GX_LAUNCHED();
    return o;
}

}  // namespace gx

namespace gx {

// Scratch-carved form of exclusive_scan_i64: the per-tile sums and prefixes
// of every level come from `scratch` (scan_scratch_bytes(n) bytes), so the
// scan itself allocates nothing.  Same kernels, same results.
size_t scan_scratch_bytes(int64_t n) {
    size_t b = 0;
    while (n > 0) {
        int64_t t = ceil_div(n, SCAN_TILE);
        b += (((size_t)t * 8 + 255) & ~size_t(255)) + (((size_t)(t + 1) * 8 + 255) & ~size_t(255));
        if (t == 1) break;
        n = t;
    }
    return b;
}

void exclusive_scan_i64_scratch(const int64_t* in, int64_t* out, int64_t n, char* scratch, cudaStream_t s) {
    if (n <= 0) {
        fill_u64(out, 0, 1, s);
        return;
    }
    int64_t ntiles = ceil_div(n, SCAN_TILE);
    int64_t* sums = reinterpret_cast<int64_t*>(scratch);
    scratch += ((size_t)ntiles * 8 + 255) & ~size_t(255);
    int64_t* pref = reinterpret_cast<int64_t*>(scratch);
    scratch += ((size_t)(ntiles + 1) * 8 + 255) & ~size_t(255);
    k_tile_sums<<<(unsigned)ntiles, SCAN_NT, 0, s>>>(in, n, sums);
    GX_LAUNCHED();
    if (ntiles == 1) fill_u64(pref, 0, 1, s);
    else exclusive_scan_i64_scratch(sums, pref, ntiles, scratch, s);
    k_tile_scan<<<(unsigned)ntiles, SCAN_NT, 0, s>>>(in, n, pref, out);
    GX_LAUNCHED();
    k_set_last<<<1, 32, 0, s>>>(pref, ntiles, sums, out, n);
    GX_LAUNCHED();
}

}  // namespace gx
