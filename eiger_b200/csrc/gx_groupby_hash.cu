// gx_groupby_hash.cu — single-pass hash group-by.
//
// Replaces gamax::groupby::hash::groupby (src/cuda/operators/groupby/
// groupby_hash.cu:302-426).  The reference builds a cuco set of row ids,
// writes 16 B/row of row-id scratch, then re-reads it to aggregate with
// global atomics.  Here one kernel streams key + value columns once:
//   * each CTA owns a shared-memory open-addressing table (keys + one
//     accumulator lane per aggregation + a 32-bit count) that absorbs every
//     key it has room for — low cardinality and Zipf heavy hitters never
//     leave shared memory;
//   * keys that do not fit go straight to a global table of AoS records
//     (key word, count word, accumulator words — one group per 32/64/128 B,
//     sized to stay L2-resident where the group count allows);
//   * at the end each CTA merges its shared table into the global one, and a
//     compaction kernel emits [key, aggregates...].
// The group count is read back once (the reference syncs three times).
#include <algorithm>

#include "gx_agg.cuh"
#include "gx_groupby.h"

namespace gx {
namespace {

constexpr uint64_t G_EMPTY4 = ~0ull;                  // 4-byte keys: never a zero-extended key
constexpr uint64_t G_EMPTY8 = 0x8000000000000000ull;  // 8-byte keys: sentinel record catches it
constexpr uint32_t S_EMPTY4 = 0x80000000u;
constexpr uint64_t S_EMPTY8 = 0x8000000000000000ull;

struct gtable {
    uint64_t* recs;        // (cap + 1) records; record `cap` holds the key equal to the empty marker
    uint64_t mask;         // cap - 1
    int* sentinel_flag;
    int* overflow;
};

template <int KW>
__device__ __forceinline__ uint32_t key_hash(uint64_t k) {
    if (KW == 4) return fmix32((uint32_t)k);
    uint64_t h = fmix64(k);
    return (uint32_t)(h ^ (h >> 32));
}

template <int KW>
__device__ __forceinline__ uint64_t* g_find_or_insert(const gtable& t, const agg_desc& d, uint64_t kw,
                                                      uint32_t h) {
    const uint64_t EMPTY = KW == 4 ? G_EMPTY4 : G_EMPTY8;
    if (KW == 8 && kw == EMPTY) {
        if (*(volatile int*)t.sentinel_flag == 0) atomicExch(t.sentinel_flag, 1);
        return t.recs + (t.mask + 1) * d.rec_words;
    }
    uint64_t slot = h & t.mask;
    for (uint64_t p = 0; p <= t.mask; ++p) {
        uint64_t* r = t.recs + slot * d.rec_words;
        uint64_t cur = *(volatile uint64_t*)r;
        if (cur == kw) return r;
        if (cur == EMPTY) {
            unsigned long long old = atomicCAS((unsigned long long*)r, (unsigned long long)EMPTY,
                                               (unsigned long long)kw);
            if (old == EMPTY || old == kw) return r;
        }
        slot = (slot + 1) & t.mask;
    }
    atomicExch(t.overflow, 1);
    return nullptr;
}

__device__ __forceinline__ void g_update(uint64_t* r, const agg_desc& d, const uint64_t (&v)[MAX_VCOLS],
                                         unsigned long long cnt) {
    if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), cnt);
    for (int a = 0; a < d.n_acc; ++a)
        dev_::acc_atomic(r + d.acc_word0 + a, d.acc_op[a], d.acc_kind[a], dev_::pick(v, d.acc_col[a]));
}

// Shared-memory table view.  Layout: keys[S] | counts[S] (u32) | acc[A][S] (u64).
template <int KW>
struct stable {
    using kt = typename std::conditional<KW == 4, uint32_t, unsigned long long>::type;
    kt* keys;
    unsigned* counts;
    uint64_t* acc;
    int* fill;
    uint32_t mask;
    int limit;
};

template <int KW>
__device__ __forceinline__ int s_find_or_insert(const stable<KW>& t, uint64_t kw, uint32_t h) {
    using kt = typename stable<KW>::kt;
    const kt EMPTY = KW == 4 ? (kt)S_EMPTY4 : (kt)S_EMPTY8;
    kt k = (kt)kw;
    if (k == EMPTY) return -1;
    uint32_t slot = h & t.mask;
    for (uint32_t p = 0; p <= t.mask; ++p) {
        kt cur = ((volatile kt*)t.keys)[slot];
        if (cur == k) return (int)slot;
        if (cur == EMPTY) {
            if (*(volatile int*)t.fill >= t.limit) return -1;  // table closed
            kt old = atomicCAS(&t.keys[slot], EMPTY, k);
            if (old == EMPTY) {
                atomicAdd(t.fill, 1);
                return (int)slot;
            }
            if (old == k) return (int)slot;
        }
        slot = (slot + 1) & t.mask;
    }
    return -1;
}

constexpr int HGB_NT = 512;
constexpr int HGB_UNROLL = 4;

template <int KW, bool SMEM>
__global__ void __launch_bounds__(HGB_NT) k_hash_groupby(const void* __restrict__ keys, int64_t n,
                                                          int key_kind, agg_desc d, gtable g,
                                                          uint32_t s_slots) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_fill;
    stable<KW> st;
    using kt = typename stable<KW>::kt;
    if (SMEM) {
        st.keys = reinterpret_cast<kt*>(smem);
        st.counts = reinterpret_cast<unsigned*>(smem + (size_t)s_slots * KW);
        st.acc = reinterpret_cast<uint64_t*>(smem + (size_t)s_slots * (KW + 4));
        st.fill = &s_fill;
        st.mask = s_slots - 1;
        st.limit = (int)(s_slots / 2);
        const kt EMPTY = KW == 4 ? (kt)S_EMPTY4 : (kt)S_EMPTY8;
        for (uint32_t i = threadIdx.x; i < s_slots; i += HGB_NT) {
            st.keys[i] = EMPTY;
            st.counts[i] = 0;
        }
        for (int a = 0; a < d.n_acc; ++a) {
            uint64_t idv;
            int op = d.acc_op[a], kind = d.acc_kind[a];
            if (op == OP_MIN) idv = kind == VK_I ? 0x7FFFFFFFFFFFFFFFull : (kind == VK_U ? ~0ull : 0x7FF0000000000000ull);
            else if (op == OP_MAX) idv = kind == VK_I ? 0x8000000000000000ull : (kind == VK_U ? 0ull : 0xFFF0000000000000ull);
            else idv = 0;
            for (uint32_t i = threadIdx.x; i < s_slots; i += HGB_NT) st.acc[(size_t)a * s_slots + i] = idv;
        }
        if (threadIdx.x == 0) s_fill = 0;
        __syncthreads();
    }

    const int64_t tile = (int64_t)HGB_NT * HGB_UNROLL;
    for (int64_t base = blockIdx.x * tile; base < n; base += (int64_t)gridDim.x * tile) {
        uint64_t kw[HGB_UNROLL];
        uint64_t v[HGB_UNROLL][MAX_VCOLS];
#pragma unroll
        for (int u = 0; u < HGB_UNROLL; ++u) {
            int64_t i = base + u * HGB_NT + threadIdx.x;
            if (i < n) {
                if (KW == 4) kw[u] = canon32(__ldg(static_cast<const unsigned*>(keys) + i), key_kind);
                else kw[u] = canon64(__ldg(static_cast<const unsigned long long*>(keys) + i), key_kind);
#pragma unroll
                for (int c = 0; c < MAX_VCOLS; ++c)
                    if (c < d.n_cols) v[u][c] = dev_::load_lane(d.col_ptr[c], d.col_width[c], d.col_kind[c], i);
            }
        }
#pragma unroll
        for (int u = 0; u < HGB_UNROLL; ++u) {
            int64_t i = base + u * HGB_NT + threadIdx.x;
            if (i >= n) continue;
            uint32_t h = key_hash<KW>(kw[u]);
            int slot = -1;
            if (SMEM) slot = s_find_or_insert<KW>(st, kw[u], h);
            if (slot >= 0) {
                if (d.has_count) atomicAdd(&st.counts[slot], 1u);
                for (int a = 0; a < d.n_acc; ++a)
                    dev_::acc_atomic(st.acc + (size_t)a * s_slots + slot, d.acc_op[a], d.acc_kind[a],
                                     dev_::pick(v[u], d.acc_col[a]));
            } else {
                uint64_t* r = g_find_or_insert<KW>(g, d, kw[u], h);
                if (r) g_update(r, d, v[u], 1ull);
            }
        }
    }

    if (SMEM) {
        __syncthreads();
        const kt EMPTY = KW == 4 ? (kt)S_EMPTY4 : (kt)S_EMPTY8;
        for (uint32_t i = threadIdx.x; i < s_slots; i += HGB_NT) {
            kt k = st.keys[i];
            if (k == EMPTY) continue;
            uint64_t kw = (uint64_t)k;
            uint64_t* r = g_find_or_insert<KW>(g, d, kw, key_hash<KW>(kw));
            if (!r) continue;
            if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), (unsigned long long)st.counts[i]);
            for (int a = 0; a < d.n_acc; ++a)
                dev_::acc_atomic(r + d.acc_word0 + a, d.acc_op[a], d.acc_kind[a],
                                 st.acc[(size_t)a * s_slots + i]);
        }
    }
}

// Initialise `nrec` records: key word = empty, count 0, accumulators = identity.
__global__ void k_init_records(uint64_t* __restrict__ recs, int64_t nrec, int rec_words, uint64_t empty,
                               agg_desc d) {
    int64_t total = nrec * rec_words;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total;
         w += (int64_t)gridDim.x * blockDim.x) {
        int f = (int)(w % rec_words);
        uint64_t val = 0;
        if (f == 0) val = empty;
        else if (f >= d.acc_word0 && f < d.acc_word0 + d.n_acc) {
            int a = f - d.acc_word0;
            int op = d.acc_op[a], kind = d.acc_kind[a];
            if (op == OP_MIN) val = kind == VK_I ? 0x7FFFFFFFFFFFFFFFull : (kind == VK_U ? ~0ull : 0x7FF0000000000000ull);
            else if (op == OP_MAX) val = kind == VK_I ? 0x8000000000000000ull : (kind == VK_U ? 0ull : 0xFFF0000000000000ull);
        }
        recs[w] = val;
    }
}

}  // namespace

void init_records(uint64_t* recs, int64_t nrec, const agg_desc& d, uint64_t empty, cudaStream_t s) {
    if (nrec <= 0) return;
    k_init_records<<<grid_for(nrec * d.rec_words, 256, 8), 256, 0, s>>>(recs, nrec, d.rec_words, empty, d);
    GX_LAUNCHED();
}

int hash_smem_slots(const agg_desc& d, int key_width, int64_t groups_bound) {
    size_t per_slot = (size_t)key_width + 4 + 8 * (size_t)d.n_acc;
    size_t budget = 100 * 1024;  // two 512-thread CTAs per SM
    uint32_t s = 1u << 16;
    while (s > 64 && s * per_slot > budget) s >>= 1;
    if (groups_bound > 0 && groups_bound < (int64_t)s / 2) {
        uint32_t want = (uint32_t)next_pow2((uint64_t)groups_bound * 2);
        if (want < 256) want = 256;
        if (want < s) s = want;
    }
    return (int)s;
}

// Runs the hash group-by into a global table of `cap` records.
// Returns false when the table overflowed (caller retries larger).
static bool hash_groupby_run(const col& key, const agg_plan& p, uint64_t cap, int smem_mode,
                             uint32_t s_slots, int64_t out_capacity, cudaStream_t s, gx_table* out) {
    const agg_desc& d = p.d;
    int kw = size_of(key.type);
    uint64_t empty = kw == 4 ? G_EMPTY4 : G_EMPTY8;
    dbuf recs((cap + 1) * d.rec_words * sizeof(uint64_t), s);
    dbuf flags(2 * sizeof(int), s);
    GX_CUDA(cudaMemsetAsync(flags.get(), 0, 2 * sizeof(int), s));
    init_records(recs.get<uint64_t>(), (int64_t)cap + 1, d, empty, s);
    gtable g;
    g.recs = recs.get<uint64_t>();
    g.mask = cap - 1;
    g.sentinel_flag = flags.get<int>();
    g.overflow = flags.get<int>() + 1;
    int kind = vkind_of(key.type);
    if (key.n > 0) {
        size_t smem = smem_mode ? (size_t)s_slots * (kw + 4 + 8 * d.n_acc) : 0;
        int per_sm = smem_mode ? std::max(1, std::min(2, (int)((200 * 1024) / std::max<size_t>(smem, 1)))) : 4;
        int grid = grid_for(key.n, HGB_NT * HGB_UNROLL, per_sm);
        GX_PROF("hash_groupby", s);
        if (kw == 4) {
            if (smem_mode) {
                GX_CUDA(cudaFuncSetAttribute(k_hash_groupby<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                k_hash_groupby<4, true><<<grid, HGB_NT, smem, s>>>(key.data, key.n, kind, d, g, s_slots);
            } else {
                k_hash_groupby<4, false><<<grid, HGB_NT, 0, s>>>(key.data, key.n, kind, d, g, 0);
            }
        } else {
            if (smem_mode) {
                GX_CUDA(cudaFuncSetAttribute(k_hash_groupby<8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                k_hash_groupby<8, true><<<grid, HGB_NT, smem, s>>>(key.data, key.n, kind, d, g, s_slots);
            } else {
                k_hash_groupby<8, false><<<grid, HGB_NT, 0, s>>>(key.data, key.n, kind, d, g, 0);
            }
        }
        GX_LAUNCHED();
    }
    int hflags[2];
    GX_CUDA(cudaMemcpyAsync(hflags, flags.get(), sizeof(hflags), cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaStreamSynchronize(s));
    if (hflags[1]) return false;
    emit_groupby_output(p, recs.get<uint64_t>(), (int64_t)cap + 1, true, empty, (int64_t)cap,
                        flags.get<int>(), key.type, out_capacity, s, out);
    return true;
}

void hash_groupby(const col& key_in, const agg_plan& p, gx_groupby_hint* hint, cudaStream_t s,
                  gx_table* out) {
    owned_col widened;
    col key = key_in;
    if (size_of(key.type) < 4) {
        widened = widen_to_32(key, s);
        key.data = widened.buf.get();
        key.type = widened.type;
    }
    int64_t n = key.n;
    int64_t bound = std::min<int64_t>(n, hint->groups_upper_bound > 0 ? hint->groups_upper_bound : n);
    bool bound_known = hint->groups_upper_bound > 0 && hint->groups_upper_bound < n;
    if (!bound_known && n > (1 << 16)) {
        // No usable bound: size from a HyperLogLog estimate (+15% margin).
        int64_t est = ndv_estimate(key, s);
        bound = std::min<int64_t>(n, std::max<int64_t>(1024, est + est / 8 + 64));
    }
    int lf = hint->load_factor_pct > 0 ? hint->load_factor_pct : 50;
    lf = std::max(10, std::min(90, lf));
    uint64_t cap = next_pow2((uint64_t)std::max<int64_t>(64, bound * 100 / lf + 1));
    uint32_t s_slots = (uint32_t)hash_smem_slots(p.d, size_of(key.type), bound_known ? bound : -1);
    // Shared tables only pay off when they can hold a useful share of the
    // keys (low cardinality, or skew that concentrates rows on few keys).
    bool smem_mode = bound <= (int64_t)s_slots * 8;
    if (const char* e = getenv("GX_HASH_SMEM")) smem_mode = atoi(e) != 0;
    int64_t out_cap = std::min<int64_t>(n, hint->groups_upper_bound > 0 ? hint->groups_upper_bound : n);
    for (int attempt = 0; attempt < 6; ++attempt) {
        if (hash_groupby_run(key, p, cap, smem_mode, s_slots, out_cap, s, out)) return;
        cap *= 4;
    }
    fail(GX_EOVERFLOW, "hash group-by table overflow after retries");
}

}  // namespace gx
