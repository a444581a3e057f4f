// gx_core.cuh — shared host/device infrastructure of the operator core:
// status/exception plumbing for the C ABI, the stream-ordered pool
// allocator, owned columns/tables, type helpers, hashing and small device
// primitives (warp/block scans, order-preserving key images).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gx.h"

namespace gx {

// ---------------------------------------------------------------------------
// Errors. C++ code throws gx::error; the C ABI layer catches and converts to
// a gx_status plus a thread-local message (reference: std::runtime_error /
// std::bad_alloc, src/cuda/operators/groupby/groupby.cu:287-299).
// ---------------------------------------------------------------------------
struct error : std::runtime_error {
    gx_status status;
    error(gx_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] inline void fail(gx_status s, const std::string& msg) { throw error(s, msg); }
inline void require(bool ok, const std::string& msg) {
    if (!ok) fail(GX_EINVAL, msg);
}
// Longest linear-probe walk in a global hash table.  Tables run at load
// <= 1/2, where walks are a few slots long; a walk this long means the table
// is (nearly) full, so the kernel reports overflow and the host retries with
// a larger table instead of scanning the whole table for every row.
constexpr uint64_t GX_PROBE_LIMIT = 4096;
// Sets the calling thread's gx_last_error_message (gx_capi.cu).
void set_last_error(const char* msg);

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        // Clear the runtime's per-thread last error (for errors that do not
        // poison the context) so a later launch check does not report it again.
        (void)cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? GX_ENOMEM : GX_ECUDA,
             std::string(what) + " failed: " + cudaGetErrorString(e) + " at " + file + ":" +
                 std::to_string(line));
    }
}
#define GX_CUDA(call) ::gx::cuda_check((call), #call, __FILE__, __LINE__)

// Every kernel launch goes through this counter so callers can verify which
// work ran on the device (gx_kernel_launch_count).
extern std::atomic<int64_t> g_launches;
#define GX_LAUNCHED()                                          \
    do {                                                       \
        ::gx::g_launches.fetch_add(1, std::memory_order_relaxed); \
        GX_CUDA(cudaGetLastError());                           \
    } while (0)

// ---------------------------------------------------------------------------
// Optional per-kernel timing with CUDA events on the launching stream
// (gx_profile_enable / gx_profile_read).  A scope records an event pair
// around the launches it encloses when profiling is on.
// ---------------------------------------------------------------------------
extern std::atomic<int> g_profiling;
struct prof_scope {
    const char* name;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    prof_scope(const char* n, cudaStream_t st);
    ~prof_scope();
};
#define GX_PROF_CAT2(a, b) a##b
#define GX_PROF_CAT(a, b) GX_PROF_CAT2(a, b)
#define GX_PROF(name, stream) ::gx::prof_scope GX_PROF_CAT(_gx_prof_, __LINE__)(name, stream)
void prof_read(const char* name, double* total_ms, int64_t* count, bool reset);

// ---------------------------------------------------------------------------
// Device properties (cached per device).  Device ordinals at or above
// GX_MAX_DEVICES are rejected with GX_EUNSUPPORTED by dev().
// ---------------------------------------------------------------------------
constexpr int GX_MAX_DEVICES = 64;
struct device_info {
    int device = 0;
    int sm_count = 148;
    int max_smem_optin = 227 * 1024;
    int l2_bytes = 126 * 1024 * 1024;
};
const device_info& dev();

// One-time per-device set-up (kernel attributes and the like), safe to call
// from several host threads: `fn` runs on the current device until one call
// returns normally, after which the device's flag stays set.  Two threads
// may both run `fn` the first time, so `fn` must be idempotent.
struct per_device_flag {
    std::atomic<bool> set[GX_MAX_DEVICES] = {};
    template <class F>
    void once(F&& fn) {
        const int d = dev().device;
        if (set[d].load(std::memory_order_acquire)) return;
        fn();
        set[d].store(true, std::memory_order_release);
    }
};

// ---------------------------------------------------------------------------
// Stream-ordered pool allocator (cudaMallocAsync on the device's default
// pool with the release threshold raised so freed blocks stay cached).
// Replaces the reference's first-fit slab (src/cuda/memory/mem_manager.cu:33-231).
// ---------------------------------------------------------------------------
void* pool_alloc(size_t bytes, cudaStream_t s);
void pool_free(void* p, cudaStream_t s);
// A device buffer of at least `bytes` kept for the calling host thread
// between library calls (one per device and slot), grown when a call needs
// more; released when the thread exits.  For the large temporaries of one
// call (the partitioned column copies, digit counts and group records of the
// PARTITION plan): allocating them from the stream pool on every call stalled for up
// to 20 ms while the pool grew.  Safe to reuse because every library call
// returns after its device work is complete.
void* thread_scratch(int slot, size_t bytes);
constexpr int SCRATCH_SLOTS = 32;
void pool_stats(int64_t* cur, int64_t* peak);
void pool_reset_peak();

// RAII device buffer bound to a stream.
class dbuf {
public:
    dbuf() = default;
    dbuf(size_t bytes, cudaStream_t s) : s_(s), bytes_(bytes) {
        p_ = bytes ? pool_alloc(bytes, s) : nullptr;
    }
    ~dbuf() { reset(); }
    dbuf(const dbuf&) = delete;
    dbuf& operator=(const dbuf&) = delete;
    dbuf(dbuf&& o) noexcept : p_(o.p_), s_(o.s_), bytes_(o.bytes_) { o.p_ = nullptr; o.bytes_ = 0; }
    dbuf& operator=(dbuf&& o) noexcept {
        if (this != &o) { reset(); p_ = o.p_; s_ = o.s_; bytes_ = o.bytes_; o.p_ = nullptr; o.bytes_ = 0; }
        return *this;
    }
    void reset() {
        if (p_) pool_free(p_, s_);
        p_ = nullptr;
        bytes_ = 0;
    }
    void* release() { void* p = p_; p_ = nullptr; bytes_ = 0; return p; }
    // Takes ownership of a buffer this pool handed out earlier (e.g. through
    // a released gx_column).
    static dbuf adopt(void* p, size_t bytes, cudaStream_t s) {
        dbuf d;
        d.p_ = p;
        d.s_ = s;
        d.bytes_ = bytes;
        return d;
    }
    template <typename T = void>
    T* get() const { return static_cast<T*>(p_); }
    size_t bytes() const { return bytes_; }

private:
    void* p_ = nullptr;
    cudaStream_t s_ = nullptr;
    size_t bytes_ = 0;
};

// ---------------------------------------------------------------------------
// Types.
// ---------------------------------------------------------------------------
inline int size_of(int t) {
    switch (t) {
        case GX_INT8: case GX_UINT8: case GX_BOOL8: return 1;
        case GX_INT16: case GX_UINT16: return 2;
        case GX_INT32: case GX_UINT32: case GX_FLOAT32: return 4;
        case GX_INT64: case GX_UINT64: case GX_FLOAT64: return 8;
        default: return 0;
    }
}
inline bool is_signed_int(int t) { return t == GX_INT8 || t == GX_INT16 || t == GX_INT32 || t == GX_INT64; }
inline bool is_unsigned_int(int t) {
    return t == GX_UINT8 || t == GX_UINT16 || t == GX_UINT32 || t == GX_UINT64 || t == GX_BOOL8;
}
inline bool is_float(int t) { return t == GX_FLOAT32 || t == GX_FLOAT64; }
inline bool is_numeric(int t) { return size_of(t) > 0; }
std::string type_name(int t);

// Value "kind" used inside kernels: how raw bits widen to a 64-bit lane.
enum vkind : int { VK_I = 0, VK_U = 1, VK_F = 2 };
inline int vkind_of(int t) { return is_float(t) ? VK_F : (is_signed_int(t) ? VK_I : VK_U); }

// A resolved column: base pointer already advanced by the view offset.
struct col {
    const void* data = nullptr;
    int64_t n = 0;
    int type = GX_EMPTY;
    template <typename T>
    const T* as() const { return static_cast<const T*>(data); }
};
inline col resolve(const gx_column_view& v) {
    col c;
    c.type = v.type;
    c.n = v.size;
    int w = size_of(v.type);
    c.data = v.data ? static_cast<const char*>(v.data) + v.offset * (int64_t)(w ? w : 1) : nullptr;
    require(v.size >= 0, "negative column size");
    require(v.offset >= 0, "negative column offset");
    return c;
}

// ---------------------------------------------------------------------------
// Owned columns / tables returned through the C ABI.
// ---------------------------------------------------------------------------
// A STRING column owns one buffer: the rows + 1 int64 offsets followed by
// the characters (ARROW layout); `str` is the host-side pair of device
// pointers that views of the column point to.
struct owned_col {
    dbuf buf;
    int64_t size = 0;
    int type = GX_EMPTY;
    bool present = true;
    std::unique_ptr<gx_string_columns> str;
};

}  // namespace gx

struct gx_table {
    std::vector<gx::owned_col> cols;
};

namespace gx {

inline owned_col make_col(int type, int64_t rows, cudaStream_t s, int64_t capacity_rows = -1) {
    owned_col c;
    c.type = type;
    c.size = rows;
    int64_t cap = capacity_rows < 0 ? rows : capacity_rows;
    size_t bytes = (size_t)cap * size_of(type);
    if (bytes) c.buf = dbuf(bytes, s);
    return c;
}
// STRING column of `rows` strings holding `char_bytes` characters in total.
inline owned_col make_string_col(int64_t rows, int64_t char_bytes, cudaStream_t s) {
    owned_col c;
    c.type = GX_STRING;
    c.size = rows;
    const size_t off_bytes = (size_t)(rows + 1) * 8;
    c.buf = dbuf(off_bytes + (size_t)std::max<int64_t>(char_bytes, 1), s);
    c.str.reset(new gx_string_columns{c.buf.get<char>() + off_bytes, c.buf.get<int64_t>()});
    return c;
}
inline gx_column to_gx_column(owned_col&& c) {
    gx_column out;
    out.size = c.size;
    out.type = c.type;
    out.capacity_bytes = (int64_t)c.buf.bytes();
    out.data = c.buf.release();
    return out;
}

// ---------------------------------------------------------------------------
// Hashing: MurmurHash3 fmix32/fmix64 finalizers (public algorithm; the
// reference uses the same finalizers for partition ids,
// src/cuda/operators/groupby/groupby_partition.cu:64-89).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t x) {
    x ^= x >> 16; x *= 0x85ebca6bU; x ^= x >> 13; x *= 0xc2b2ae35U; x ^= x >> 16;
    return x;
}
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}

// Canonical equality image of a key's raw bits: float -0.0 and +0.0 compare
// equal (the reference compares keys with operator==), so they map to the
// same bits.  `kind`: VK_I/VK_U keep the bits, VK_F normalises zero.
__host__ __device__ __forceinline__ uint32_t canon32(uint32_t b, int kind) {
    return (kind == VK_F && (b << 1) == 0u) ? 0u : b;
}
__host__ __device__ __forceinline__ uint64_t canon64(uint64_t b, int kind) {
    return (kind == VK_F && (b << 1) == 0ull) ? 0ull : b;
}

// Order-preserving unsigned image of a key (radix sort digit source):
// signed ints flip the sign bit, floats flip all bits when negative and the
// sign bit otherwise (-0.0 first normalised to +0.0), unsigned unchanged.
__host__ __device__ __forceinline__ uint32_t ordered32(uint32_t b, int kind) {
    if (kind == VK_I) return b ^ 0x80000000u;
    if (kind == VK_F) {
        if (b == 0x80000000u) b = 0u;
        return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    }
    return b;
}
__host__ __device__ __forceinline__ uint64_t ordered64(uint64_t b, int kind) {
    if (kind == VK_I) return b ^ 0x8000000000000000ull;
    if (kind == VK_F) {
        if (b == 0x8000000000000000ull) b = 0ull;
        return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
    }
    return b;
}

// Radix-sort digit source: the order-preserving image of a key (narrow keys
// widened to 4 bytes carry their logical width), inverted for a descending
// sort, minus a bias (a sort on the bits the keys span).
struct img_params {
    int kind;      // vkind of the key type
    int lw;        // logical key width in bytes (1, 2, 4, 8)
    int desc;      // descending
    uint64_t bias; // subtracted from the image before digit extraction
};

template <int KW>
__host__ __device__ __forceinline__ uint64_t key_image(uint64_t raw, const img_params& ip) {
    uint64_t img;
    if (KW == 4) {
        uint32_t b = (uint32_t)raw;
        if (ip.lw < 4) {
            b &= (1u << (8 * ip.lw)) - 1u;
            if (ip.kind == VK_I) b ^= 1u << (8 * ip.lw - 1);
        } else {
            b = ordered32(b, ip.kind);
        }
        img = b;
        if (ip.desc) img = (~img) & 0xFFFFFFFFull;
    } else {
        img = ordered64(raw, ip.kind);
        if (ip.desc) img = ~img;
    }
    return img - ip.bias;
}

// ---------------------------------------------------------------------------
// Small helpers.
// ---------------------------------------------------------------------------
inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int ilog2_ceil(uint64_t x) {
    int b = 0;
    while ((uint64_t(1) << b) < x) ++b;
    return b;
}
inline uint64_t next_pow2(uint64_t x) { return x <= 1 ? 1 : (uint64_t(1) << ilog2_ceil(x)); }
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Host <- device copy of a small value with a stream sync.
template <typename T>
T read_scalar(const T* dptr, cudaStream_t s) {
    T v;
    GX_CUDA(cudaMemcpyAsync(&v, dptr, sizeof(T), cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaStreamSynchronize(s));
    return v;
}

// Grid size for a grid-stride kernel: a multiple of the SM count.
inline int grid_for(int64_t work_items, int per_block, int blocks_per_sm = 4) {
    int64_t need = ceil_div(work_items > 0 ? work_items : 1, per_block);
    int64_t cap = (int64_t)dev().sm_count * blocks_per_sm;
    return (int)(need < cap ? need : cap);
}

// Fill a device buffer of 8-byte words with a pattern (kernel in gx_util.cu).
void fill_u64(void* dst, uint64_t pattern, int64_t words, cudaStream_t s);
void fill_u32(void* dst, uint32_t pattern, int64_t words, cudaStream_t s);
// Exclusive scan of int64 counts into offsets (n+1 outputs, out[n] = total).
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);
// The same scan with its temporaries carved from caller scratch.
size_t scan_scratch_bytes(int64_t n);
void exclusive_scan_i64_scratch(const int64_t* in, int64_t* out, int64_t n, char* scratch, cudaStream_t s);
// iota of int64.
void sequence_i64(int64_t* out, int64_t n, int64_t start, int64_t step, cudaStream_t s);
// out[i] = src[idx[i]] for `width`-byte elements.
void gather_bytes(void* out, const void* src, const int64_t* idx, int64_t n, int width,
                  cudaStream_t s);
// Widen a 1/2-byte integer column to 4 bytes (sign- or zero-extended).
owned_col widen_to_32(const col& c, cudaStream_t s);

}  // namespace gx

// ---------------------------------------------------------------------------
// Device-side helpers.
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
namespace gx {
namespace dev_ {

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Inclusive warp scan.
template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane_id() >= o) v += n;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide exclusive scan for blockDim.x == NT (multiple of 32).
// `smem` needs NT/32 + 1 slots.  Returns exclusive prefix; *total gets the sum.
template <int NT, typename T>
__device__ __forceinline__ T block_exclusive_sum(T v, T* smem, T* total) {
    const int warp = threadIdx.x >> 5;
    T inc = warp_inclusive_sum(v);
    if (lane_id() == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane_id() < NT / 32 ? smem[lane_id()] : T(0);
        T wi = warp_inclusive_sum(w);
        if (lane_id() < NT / 32) smem[lane_id()] = wi - w;
        if (lane_id() == NT / 32 - 1) smem[NT / 32] = wi;
    }
    __syncthreads();
    T res = smem[warp] + inc - v;
    *total = smem[NT / 32];
    __syncthreads();
    return res;
}

// ---- Bulk global -> shared copies (the copy engine behind TMA) completed on
// an mbarrier.  Addresses are shared-window offsets.  Both ends of a copy must
// be 16-byte aligned and its size a multiple of 16; one barrier phase may
// expect at most 2^20 - 1 bytes.
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(arrivals) : "memory");
}
// Makes barrier initialisation visible to the copy engine (async proxy).
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// One arrival that also announces `bytes` of incoming copy traffic.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the barrier phase with the given parity to complete, giving up
// after `limit` polls (each poll may suspend the thread for a short,
// hardware-chosen time).  Returns false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace dev_
}  // namespace gx
#endif
