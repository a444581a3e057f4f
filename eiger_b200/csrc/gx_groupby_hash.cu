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
#include "gx_groupby_hash_spec.cuh"

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
    for (uint64_t p = 0, lim = t.mask < GX_PROBE_LIMIT ? t.mask : GX_PROBE_LIMIT - 1; p <= lim; ++p) {
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

template <int NV>
__device__ __forceinline__ void g_update(uint64_t* r, const agg_desc& d, const uint64_t (&v)[NV],
                                         unsigned long long cnt) {
    if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), cnt);
    for (int a = 0; a < d.n_acc; ++a) {
        const int op = d.acc_op[a], kind = d.acc_kind[a];
        const uint64_t x = dev_::pick(v, d.acc_col[a]);
        uint64_t* p = r + d.acc_word0 + a;
        if (op == OP_MIN || op == OP_MAX) {
            // A plain (possibly stale) read first: extremes only tighten, so a
            // stale value can only cause an unneeded atomic, never a lost one.
            if (!dev_::improves(op, kind, x, *p)) continue;
        }
        dev_::acc_atomic(p, op, kind, x);
    }
}

// Shared-memory table of one CTA:
//   keys[S] (u32 or u64) | counts[S][R] (u32) | acc[A][S][R] (u64)
// The key table is shared by the CTA; the accumulators are replicated R
// times (thread t updates replica t % R) so that low-cardinality inputs do
// not serialise on a handful of shared-memory words.  Replicas are the
// innermost index: with R = 32 the lanes of a warp update 32 different
// banks whatever slots they hit (R = 16: conflict-free 8-byte updates).
template <int KW>
struct stable {
    using kt = typename std::conditional<KW == 4, uint32_t, unsigned long long>::type;
    kt* keys;
    unsigned* counts;
    uint64_t* acc;
    int* fill;
    uint32_t mask;
    int limit;
    uint32_t S;
    int R;
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

constexpr int HGB_NT = 1024;
constexpr int64_t HASH_UNITS_MAX_GROUPS = 4096;
constexpr int HGB_UNROLL = 4;
// Rows per thread per batch in the unit kernels: three measured best for the
// dense-id kernel (7 aggregates at 2^28 rows, 2^16 groups: 2.52 ms against
// 2.60 with two and 2.98 with four).
constexpr int HU_UNROLL = 3;

template <int KW, bool SMEM, int NV, class... ACCS>
__global__ void __launch_bounds__(HGB_NT, 1) k_hash_groupby(const void* __restrict__ keys, int64_t n,
                                                             int key_kind, agg_desc d, gtable g,
                                                             uint32_t s_slots, int reps) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_fill;
    // Per-warp queue of a batch's rows whose key was not at its home slot.
    __shared__ unsigned short s_bq[SMEM ? HGB_NT / 32 : 1][SMEM ? 32 * HGB_UNROLL : 1];
    stable<KW> st;
    using kt = typename stable<KW>::kt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    unsigned* my_counts = nullptr;
    uint64_t* my_acc = nullptr;
    if (SMEM) {
        const size_t S = s_slots;
        const size_t key_bytes = (S * KW + 15) & ~size_t(15);
        st.keys = reinterpret_cast<kt*>(smem);
        st.counts = reinterpret_cast<unsigned*>(smem + key_bytes);
        st.acc = reinterpret_cast<uint64_t*>(smem + key_bytes + ((S * 4 * reps + 15) & ~size_t(15)));
        st.fill = &s_fill;
        st.mask = s_slots - 1;
        st.limit = (int)(s_slots / 2);
        st.S = s_slots;
        st.R = reps;
        const kt EMPTY = KW == 4 ? (kt)S_EMPTY4 : (kt)S_EMPTY8;
        for (uint32_t i = threadIdx.x; i < s_slots; i += HGB_NT) st.keys[i] = EMPTY;
        for (uint32_t i = threadIdx.x; i < s_slots * reps; i += HGB_NT) st.counts[i] = 0;
        for (int a = 0; a < d.n_acc; ++a) {
            uint64_t idv = dev_::acc_ident(d.acc_op[a], d.acc_kind[a]);
            uint64_t* base = st.acc + (size_t)a * S * reps;
            for (uint32_t i = threadIdx.x; i < s_slots * reps; i += HGB_NT) base[i] = idv;
        }
        if (threadIdx.x == 0) s_fill = 0;
        // Spread a warp's lanes over the replicas: lanes of one warp that hit
        // the same group then update different words.
        const int rep = (int)(threadIdx.x % (unsigned)reps);
        my_counts = st.counts + rep;
        my_acc = st.acc + rep;
        __syncthreads();
    }

    const int64_t tile = (int64_t)HGB_NT * HGB_UNROLL;
    for (int64_t base = blockIdx.x * tile; base < n; base += (int64_t)gridDim.x * tile) {
        uint64_t kw[HGB_UNROLL];
        uint64_t v[HGB_UNROLL][NV];
#pragma unroll
        for (int u = 0; u < HGB_UNROLL; ++u) {
            int64_t i = base + u * HGB_NT + threadIdx.x;
            if (i < n) {
                if (KW == 4) kw[u] = canon32(__ldg(static_cast<const unsigned*>(keys) + i), key_kind);
                else kw[u] = canon64(__ldg(static_cast<const unsigned long long*>(keys) + i), key_kind);
                if constexpr (sizeof...(ACCS) > 0) {
#pragma unroll
                    for (int c = 0; c < NV; ++c)
                        v[u][c] = __ldg(static_cast<const unsigned long long*>(d.col_ptr[c]) + i);
                } else {
#pragma unroll
                    for (int c = 0; c < NV; ++c)
                        if (c < d.n_cols) v[u][c] = dev_::load_lane(d.col_ptr[c], d.col_width[c], d.col_kind[c], i);
                }
            }
        }
        if constexpr (SMEM) {
            // Home-slot probe of every row of the batch at once; rows found
            // there update now, the others are queued (offset in the batch)
            // and walk the probe sequence together at the end of the batch.
            const kt EMPTY = KW == 4 ? (kt)S_EMPTY4 : (kt)S_EMPTY8;
            int qfill = 0;
#pragma unroll
            for (int u = 0; u < HGB_UNROLL; ++u) {
                const int off = u * HGB_NT + (int)threadIdx.x;
                const bool valid = base + off < n;
                const uint32_t h = valid ? key_hash<KW>(kw[u]) : 0u;
                int slot = -2;
                if (valid && (kt)kw[u] != EMPTY) {
                    const uint32_t s0 = h & st.mask;
                    if (((volatile kt*)st.keys)[s0] == (kt)kw[u]) slot = (int)s0;
                }
                const bool miss = valid && slot == -2;
                const unsigned mm = __ballot_sync(0xffffffffu, miss);
                if (miss) s_bq[warp][qfill + __popc(mm & lt)] = (unsigned short)off;
                qfill += __popc(mm);
                if (valid && slot >= 0) {
                    // The per-replica count is kept even without COUNT: it
                    // tells the merge which replicas saw the group (for ANY).
                    atomicAdd(&my_counts[slot * reps], 1u);
                    if constexpr (sizeof...(ACCS) > 0) spec::apply_all<0, ACCS...>(my_acc, s_slots * reps, slot * reps, v[u]);
                    else dev_::shared_row_update<NV>(my_acc, (size_t)s_slots * reps, slot * reps, d, v[u]);
                }
            }
            __syncwarp();
            for (int q0 = 0; q0 < qfill; q0 += 32) {
                const bool live = q0 + lane < qfill;
                const int64_t i = base + (live ? s_bq[warp][q0 + lane] : 0);
                uint64_t kq = 0, vq[NV];
                if (live) {
                    if (KW == 4) kq = canon32(__ldg(static_cast<const unsigned*>(keys) + i), key_kind);
                    else kq = canon64(__ldg(static_cast<const unsigned long long*>(keys) + i), key_kind);
                    if constexpr (sizeof...(ACCS) > 0) {
#pragma unroll
                        for (int c = 0; c < NV; ++c) vq[c] = __ldg(static_cast<const unsigned long long*>(d.col_ptr[c]) + i);
                    } else {
#pragma unroll
                        for (int c = 0; c < NV; ++c)
                            if (c < d.n_cols) vq[c] = dev_::load_lane(d.col_ptr[c], d.col_width[c], d.col_kind[c], i);
                    }
                }
                const uint32_t hq = live ? key_hash<KW>(kq) : 0u;
                const int sq = live ? s_find_or_insert<KW>(st, kq, hq) : -1;
                // Lanes leave the probe loop at different steps; regroup the
                // warp so the updates issue once per warp, not once per exit step.
                __syncwarp();
                if (live) {
                    if (sq >= 0) {
                        atomicAdd(&my_counts[sq * reps], 1u);
                        if constexpr (sizeof...(ACCS) > 0) spec::apply_all<0, ACCS...>(my_acc, s_slots * reps, sq * reps, vq);
                        else dev_::shared_row_update<NV>(my_acc, (size_t)s_slots * reps, sq * reps, d, vq);
                    } else {
                        uint64_t* r = g_find_or_insert<KW>(g, d, kq, hq);
                        if (r) g_update(r, d, vq, 1ull);
                    }
                }
                __syncwarp();
            }
        } else {
#pragma unroll
            for (int u = 0; u < HGB_UNROLL; ++u) {
                const int64_t i = base + u * HGB_NT + threadIdx.x;
                if (i >= n) continue;
                const uint32_t h = key_hash<KW>(kw[u]);
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
            unsigned long long c = 0;
            int first = -1;
            for (int rp = 0; rp < reps; ++rp) {
                unsigned cr = st.counts[(size_t)i * reps + rp];
                c += cr;
                if (cr && first < 0) first = rp;
            }
            if (first < 0) continue;
            if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), c);
            for (int a = 0; a < d.n_acc; ++a) {
                uint64_t x = st.acc[((size_t)a * s_slots + i) * reps + first];
                for (int rp = first + 1; rp < reps; ++rp)
                    if (st.counts[(size_t)i * reps + rp])
                        x = dev_::acc_combine(d.acc_op[a], d.acc_kind[a], x,
                                              st.acc[((size_t)a * s_slots + i) * reps + rp]);
                dev_::acc_atomic(r + d.acc_word0 + a, d.acc_op[a], d.acc_kind[a], x);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Aggregation of radix-partitioned rows, one work unit at a time.  A unit is
// a row range of one partition, so it holds only that partition's groups and
// the CTA's shared table (sized for them) absorbs every row; the shared-table
// update is the same code as k_hash_groupby's.  The table slot comes from the
// hash bits above the partition bits.  A unit that is a whole partition and
// never overflowed its table appends its final groups densely; a split (or
// spilled) unit merges into the global table like k_hash_groupby's CTAs.
// ---------------------------------------------------------------------------
template <int KW, int NV, class... ACCS>
__global__ void __launch_bounds__(HGB_NT, 1) k_hash_units(const void* __restrict__ keys, int key_kind, agg_desc d,
                                                           const part_unit* __restrict__ units,
                                                           const int64_t* __restrict__ n_units, uint32_t s_slots,
                                                           int reps, int shift, gtable g,
                                                           uint64_t* __restrict__ out_recs,
                                                           unsigned long long* __restrict__ out_count,
                                                           int64_t rec_cap, int* __restrict__ rec_ovf) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_fill, s_spill;
    __shared__ unsigned long long s_base;
    __shared__ int64_t scan_sm[HGB_NT / 32 + 1];
    // Per-warp queue of rows whose key was not at its home slot: at most 31
    // left over plus HU_UNROLL × 32 from one batch.
    __shared__ uint32_t s_q[HGB_NT / 32][31 + 32 * HU_UNROLL];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    using kt = typename stable<KW>::kt;
    const kt EMPTY = KW == 4 ? (kt)S_EMPTY4 : (kt)S_EMPTY8;
    stable<KW> st;
    const size_t S = s_slots;
    const size_t key_bytes = (S * KW + 15) & ~size_t(15);
    st.keys = reinterpret_cast<kt*>(smem);
    st.counts = reinterpret_cast<unsigned*>(smem + key_bytes);
    st.acc = reinterpret_cast<uint64_t*>(smem + key_bytes + ((S * 4 * reps + 15) & ~size_t(15)));
    st.fill = &s_fill;
    st.mask = s_slots - 1;
    st.limit = (int)(s_slots / 2);
    st.S = s_slots;
    st.R = reps;
    const int rep = (int)(threadIdx.x % (unsigned)reps);
    unsigned* my_counts = st.counts + rep;
    uint64_t* my_acc = st.acc + rep;
    const int64_t nu = *n_units;
    for (int64_t u = blockIdx.x; u < nu; u += gridDim.x) {
        const part_unit un = units[u];
        for (uint32_t i = threadIdx.x; i < s_slots; i += HGB_NT) st.keys[i] = EMPTY;
        for (uint32_t i = threadIdx.x; i < s_slots * reps; i += HGB_NT) st.counts[i] = 0;
        for (int a = 0; a < d.n_acc; ++a) {
            const uint64_t idv = dev_::acc_ident(d.acc_op[a], d.acc_kind[a]);
            uint64_t* base = st.acc + (size_t)a * S * reps;
            for (uint32_t i = threadIdx.x; i < s_slots * reps; i += HGB_NT) base[i] = idv;
        }
        if (threadIdx.x == 0) { s_fill = 0; s_spill = 0; }
        __syncthreads();
        const int64_t tile = (int64_t)HGB_NT * HU_UNROLL;
        // One queued row per lane: load it again (cached), walk its probe
        // sequence, update (or spill to the global table).
        auto drain = [&](uint32_t off, bool live) {
            const int64_t i = un.begin + off;
            uint64_t kq = 0, vq[NV];
            if (live) {
                if (KW == 4) kq = canon32(__ldg(static_cast<const unsigned*>(keys) + i), key_kind);
                else kq = canon64(__ldg(static_cast<const unsigned long long*>(keys) + i), key_kind);
                if constexpr (sizeof...(ACCS) > 0) {
#pragma unroll
                    for (int c = 0; c < NV; ++c) vq[c] = __ldg(static_cast<const unsigned long long*>(d.col_ptr[c]) + i);
                } else {
#pragma unroll
                    for (int c = 0; c < NV; ++c)
                        if (c < d.n_cols) vq[c] = dev_::load_lane(d.col_ptr[c], d.col_width[c], d.col_kind[c], i);
                }
            }
            const uint32_t hq = live ? key_hash<KW>(kq) : 0u;
            const int sq = live ? s_find_or_insert<KW>(st, kq, hq >> shift) : -1;
            __syncwarp();  // regroup after the probe loop (see k_hash_groupby)
            if (!live) return;
            if (sq >= 0) {
                atomicAdd(&my_counts[sq * reps], 1u);
                if constexpr (sizeof...(ACCS) > 0) spec::apply_all<0, ACCS...>(my_acc, s_slots * reps, sq * reps, vq);
                else dev_::shared_row_update<NV>(my_acc, (size_t)s_slots * reps, sq * reps, d, vq);
            } else {
                if (!s_spill) s_spill = 1;
                uint64_t* r = g_find_or_insert<KW>(g, d, kq, hq);
                if (r) g_update(r, d, vq, 1ull);
            }
        };
        int qfill = 0;
        for (int64_t base = un.begin; base < un.end; base += tile) {
            uint64_t kw[HU_UNROLL];
            uint64_t v[HU_UNROLL][NV];
#pragma unroll
            for (int q = 0; q < HU_UNROLL; ++q) {
                const int64_t i = base + q * HGB_NT + threadIdx.x;
                if (i < un.end) {
                    if (KW == 4) kw[q] = canon32(__ldg(static_cast<const unsigned*>(keys) + i), key_kind);
                    else kw[q] = canon64(__ldg(static_cast<const unsigned long long*>(keys) + i), key_kind);
                    if constexpr (sizeof...(ACCS) > 0) {
#pragma unroll
                        for (int c = 0; c < NV; ++c)
                            v[q][c] = __ldg(static_cast<const unsigned long long*>(d.col_ptr[c]) + i);
                    } else {
#pragma unroll
                        for (int c = 0; c < NV; ++c)
                            if (c < d.n_cols) v[q][c] = dev_::load_lane(d.col_ptr[c], d.col_width[c], d.col_kind[c], i);
                    }
                }
            }
            // First probe of every row of the batch at once (independent
            // shared loads); only a row whose home slot holds another key
            // (or is empty) walks the probe sequence.
            uint32_t h[HU_UNROLL];
            int slot[HU_UNROLL];
#pragma unroll
            for (int q = 0; q < HU_UNROLL; ++q) {
                const bool valid = base + q * HGB_NT + threadIdx.x < un.end;
                h[q] = valid ? key_hash<KW>(kw[q]) : 0u;
                slot[q] = -2;
                if (valid && (kt)kw[q] != EMPTY) {
                    const uint32_t s0 = (h[q] >> shift) & st.mask;
                    if (((volatile kt*)st.keys)[s0] == (kt)kw[q]) slot[q] = (int)s0;
                }
            }
            // Rows found at home update now; the others are queued (row
            // offset in the unit) and walk the probe sequence later, 32 at a
            // time with every lane busy, instead of holding the whole warp in
            // a loop for one or two lanes.
#pragma unroll
            for (int q = 0; q < HU_UNROLL; ++q) {
                const int64_t i = base + q * HGB_NT + threadIdx.x;
                const bool valid = i < un.end;
                const bool miss = valid && slot[q] == -2;
                const unsigned mm = __ballot_sync(0xffffffffu, miss);
                if (miss) s_q[warp][qfill + __popc(mm & lt)] = (uint32_t)(i - un.begin);
                qfill += __popc(mm);
                if (valid && slot[q] >= 0) {
                    atomicAdd(&my_counts[slot[q] * reps], 1u);
                    if constexpr (sizeof...(ACCS) > 0) spec::apply_all<0, ACCS...>(my_acc, s_slots * reps, slot[q] * reps, v[q]);
                    else dev_::shared_row_update<NV>(my_acc, (size_t)s_slots * reps, slot[q] * reps, d, v[q]);
                }
            }
            __syncwarp();
            while (qfill >= 32) {
                qfill -= 32;
                drain(s_q[warp][qfill + lane], true);
            }
        }
        drain(lane < qfill ? s_q[warp][lane] : 0u, lane < qfill);
        qfill = 0;
        __syncthreads();
        const bool final_groups = !un.split && !s_spill;
        if (final_groups) {
            if (threadIdx.x == 0) {
                s_base = atomicAdd(out_count, (unsigned long long)s_fill);
                if ((int64_t)(s_base + s_fill) > rec_cap) atomicExch(rec_ovf, 1);
            }
            __syncthreads();
        }
        if (final_groups && (int64_t)(s_base + s_fill) <= rec_cap) {
            // Compact the occupied slots (slot order) into dense records.
            int64_t running = 0;
            for (uint32_t i0 = 0; i0 < s_slots; i0 += HGB_NT) {
                const uint32_t i = i0 + threadIdx.x;
                const bool live = i < s_slots && st.keys[i] != EMPTY;
                int64_t tot;
                const int64_t ex = dev_::block_exclusive_sum<HGB_NT, int64_t>(live ? 1 : 0, scan_sm, &tot);
                if (live) {
                    uint64_t* r = out_recs + (s_base + running + ex) * d.rec_words;
                    unsigned long long c = 0;
                    int first = -1;
                    for (int rp = 0; rp < reps; ++rp) {
                        const unsigned cr = st.counts[(size_t)i * reps + rp];
                        c += cr;
                        if (cr && first < 0) first = rp;
                    }
                    r[0] = (uint64_t)st.keys[i];
                    if (d.has_count) r[d.count_word] = c;
                    for (int a = 0; a < d.n_acc; ++a) {
                        uint64_t x = dev_::acc_ident(d.acc_op[a], d.acc_kind[a]);
                        if (first >= 0) {
                            x = st.acc[((size_t)a * S + i) * reps + first];
                            for (int rp = first + 1; rp < reps; ++rp)
                                if (st.counts[(size_t)i * reps + rp])
                                    x = dev_::acc_combine(d.acc_op[a], d.acc_kind[a], x,
                                                          st.acc[((size_t)a * S + i) * reps + rp]);
                        }
                        r[d.acc_word0 + a] = x;
                    }
                }
                running += tot;
            }
        } else if (!final_groups) {
            for (uint32_t i = threadIdx.x; i < s_slots; i += HGB_NT) {
                const kt k = st.keys[i];
                if (k == EMPTY) continue;
                const uint64_t kwv = (uint64_t)k;
                uint64_t* r = g_find_or_insert<KW>(g, d, kwv, key_hash<KW>(kwv));
                if (!r) continue;
                unsigned long long c = 0;
                int first = -1;
                for (int rp = 0; rp < reps; ++rp) {
                    const unsigned cr = st.counts[(size_t)i * reps + rp];
                    c += cr;
                    if (cr && first < 0) first = rp;
                }
                if (first < 0) continue;
                if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), c);
                for (int a = 0; a < d.n_acc; ++a) {
                    uint64_t x = st.acc[((size_t)a * S + i) * reps + first];
                    for (int rp = first + 1; rp < reps; ++rp)
                        if (st.counts[(size_t)i * reps + rp])
                            x = dev_::acc_combine(d.acc_op[a], d.acc_kind[a], x,
                                                  st.acc[((size_t)a * S + i) * reps + rp]);
                    dev_::acc_atomic(r + d.acc_word0 + a, d.acc_op[a], d.acc_kind[a], x);
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Unit aggregation with dense group ids (compiled plans, or the run-time
// aggregation list with up to four value columns of any width).
//
// k_hash_units indexes its accumulators by table slot, and at the load its
// tables run at (<= 1/4) the slots leave room for one accumulator replica.
// Here the CTA hands out dense group ids in insertion order and indexes the
// accumulators by id, R replicas innermost (lane l updates replica l % R):
// sized by groups instead of slots, 8 replicas fit at ~256 groups per
// partition with 7 aggregates (2.92 -> 2.60 ms at 2^28 rows, G = 2^16).
//
// Slot words: 4-byte keys pack key << 32 | id, so the probe is one load and
// one compare.  8-byte keys pack id << 32 | 32-bit key hash and keep the key
// itself in gkey[id]; a row whose hash matches confirms the key there, and a
// different key with the same hash simply continues the probe walk.
//
// Insertion claims an empty slot (id PENDING), takes the next id, writes
// the key of the id and publishes the slot word.  A row that finds its slot
// PENDING (or, for 8-byte keys, the id's key not yet visible) retries with
// its whole warp after the warp regroups, a bounded number of rounds; when
// the rounds, the ids (gcap) or the probe walk run out, the row goes to the
// global table and the unit is merged there instead of appended.  The
// replicas a unit uses are chosen per unit (all for a piece of a split
// partition, one per 16 rows of a group otherwise).
// ---------------------------------------------------------------------------
constexpr unsigned long long UD_EMPTY = ~0ull;
constexpr uint32_t UD_PENDING = 0xFFFFFFFEu;
constexpr uint32_t UD_SPILL = 0xFFFFFFFDu;
constexpr uint32_t UD_WAIT_LIMIT = 1u << 16;

// Slot word accesses (single 8-byte loads and stores).  For 8-byte keys
// gkey[] holds UD_UNSET from the start of each unit until an id's key is
// written (each id is written once per unit), so a read of gkey[id] yields
// either UD_UNSET or the id's true key: a reader that matches its key there
// has found its group whatever order the two writes became visible in, and
// one that reads UD_UNSET waits for the key (bounded).  Keys equal to
// UD_UNSET go to the global table.  No fence or acquire load is needed on
// the row path (acquire loads there cost 2.6x at 2^24 groups: they also
// order the row's earlier value loads).
constexpr unsigned long long UD_UNSET = 0x8000000000000000ull;
template <int KW>
__device__ __forceinline__ unsigned long long ld_slot(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
template <int KW>
__device__ __forceinline__ void st_slot(unsigned long long* p, unsigned long long v) {
    *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

template <int KW>
struct dtable {
    using kt = typename std::conditional<KW == 4, uint32_t, unsigned long long>::type;
    unsigned long long* slots;  // [S] slot words (see above)
    kt* gkey;                   // [gcap] key of each group id
    int* fill;                  // ids handed out
    uint32_t mask, gcap;
};

// Slot word layout per key width: the id and the tag to compare.
template <int KW>
__device__ __forceinline__ uint32_t ud_id(unsigned long long w) {
    return KW == 4 ? (uint32_t)w : (uint32_t)(w >> 32);
}
template <int KW>
__device__ __forceinline__ uint32_t ud_tag(unsigned long long w) {
    return KW == 4 ? (uint32_t)(w >> 32) : (uint32_t)w;
}
template <int KW>
__device__ __forceinline__ unsigned long long ud_word(uint32_t tag, uint32_t id) {
    return KW == 4 ? ((unsigned long long)tag << 32) | id : ((unsigned long long)id << 32) | tag;
}

// Group id of key k (canonical; tag = the key itself for 4-byte keys, its
// 32-bit hash for 8-byte ones), inserting it.  Returns UD_PENDING when the
// key's slot is claimed but not yet published (or, for 8-byte keys, its id's
// key is not yet visible) instead of waiting: the inserter may be a lane of
// the same warp, which a spinning branch can hold back.  UD_SPILL when the
// ids or the probe walk run out.
template <int KW>
__device__ __forceinline__ uint32_t d_find_or_insert(const dtable<KW>& t, uint64_t k, uint32_t tag, uint32_t h) {
    if (KW == 8 && k == UD_UNSET) return UD_SPILL;
    uint32_t slot = h & t.mask;
    for (uint32_t p = 0; p <= t.mask; ++p) {
        unsigned long long cur = ld_slot<KW>(&t.slots[slot]);
        if (cur == UD_EMPTY) {
            cur = atomicCAS(&t.slots[slot], UD_EMPTY, ud_word<KW>(tag, UD_PENDING));
            if (cur == UD_EMPTY) {
                uint32_t g = (uint32_t)atomicAdd(t.fill, 1);
                if (g < t.gcap) t.gkey[g] = (typename dtable<KW>::kt)k;
                else g = UD_SPILL;
                st_slot<KW>(&t.slots[slot], ud_word<KW>(tag, g));
                return g;
            }
        }
        if (ud_tag<KW>(cur) == tag) {
            const uint32_t g = ud_id<KW>(cur);
            if (g == UD_PENDING || g == UD_SPILL) return g;
            if (KW == 4) return g;
            const unsigned long long kk = reinterpret_cast<volatile unsigned long long*>(t.gkey)[g];
            if (kk == UD_UNSET) return UD_PENDING;
            if (kk == k) return g;
        }
        slot = (slot + 1) & t.mask;
    }
    return UD_SPILL;
}

// d_find_or_insert for the live lanes of a whole warp (every lane calls it):
// lanes that meet a pending slot retry after the warp regroups, so an
// inserter in the same warp has published; after UD_WAIT_LIMIT rounds they
// get UD_SPILL (their rows go to the global table).  Non-live lanes return
// UD_SPILL.
template <int KW>
__device__ __forceinline__ uint32_t d_find_or_insert_warp(const dtable<KW>& t, bool live, uint64_t k, uint32_t tag,
                                                          uint32_t h) {
    uint32_t g = live ? d_find_or_insert<KW>(t, k, tag, h) : UD_SPILL;
    for (uint32_t round = 0; __any_sync(0xffffffffu, g == UD_PENDING); ++round) {
        __syncwarp();
        if (g == UD_PENDING) g = round < UD_WAIT_LIMIT ? d_find_or_insert<KW>(t, k, tag, h) : UD_SPILL;
    }
    return g;
}

template <int KW>
__device__ __forceinline__ uint64_t ud_load_key(const void* keys, int64_t i, int kind) {
    if (KW == 4) return canon32(__ldg(static_cast<const unsigned*>(keys) + i), kind);
    return canon64(__ldg(static_cast<const unsigned long long*>(keys) + i), kind);
}

template <int KW, int NV, class... ACCS>
__global__ void __launch_bounds__(HGB_NT, 1) k_units_dense(const void* __restrict__ keys, int key_kind, agg_desc d,
                                                            const part_unit* __restrict__ units,
                                                            const int64_t* __restrict__ n_units, uint32_t s_slots,
                                                            uint32_t gcap, int reps, uint32_t gpp, int shift,
                                                            gtable g, uint64_t* __restrict__ out_recs,
                                                            unsigned long long* __restrict__ out_count,
                                                            int64_t rec_cap, int* __restrict__ rec_ovf) {
    constexpr bool CP = sizeof...(ACCS) > 0;  // compiled plan: 8-byte columns, straight-line updates
    using kt = typename dtable<KW>::kt;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_fill, s_spill;
    __shared__ unsigned long long s_base;
    __shared__ uint32_t s_q[HGB_NT / 32][31 + 32 * HU_UNROLL];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int NA = CP ? (int)sizeof...(ACCS) : d.n_acc;
    const size_t GR = (size_t)gcap * reps;  // words per accumulator (layout for `reps` replicas)
    dtable<KW> t;
    t.slots = reinterpret_cast<unsigned long long*>(smem);
    t.gkey = reinterpret_cast<kt*>(smem + (size_t)s_slots * 8);
    unsigned* counts =
        reinterpret_cast<unsigned*>(smem + (size_t)s_slots * 8 + (((size_t)gcap * KW + 15) & ~size_t(15)));
    uint64_t* acc = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(counts) + ((GR * 4 + 15) & ~size_t(15)));
    t.fill = &s_fill;
    t.mask = s_slots - 1;
    t.gcap = gcap;
    // tag of a key in its slot word: the key (4 bytes) or its hash (8 bytes)
    auto tag_of = [](uint64_t k, uint32_t h) { return KW == 4 ? (uint32_t)k : h; };
    // Row i's value lanes, and one row's accumulator updates at word `at` of
    // the accumulator arrays starting at `ma`.
    auto load_vals = [&](int64_t i, uint64_t (&vv)[NV]) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            if constexpr (CP) vv[c] = __ldg(static_cast<const unsigned long long*>(d.col_ptr[c]) + i);
            else vv[c] = c < d.n_cols ? dev_::load_lane(d.col_ptr[c], d.col_width[c], d.col_kind[c], i) : 0ull;
        }
    };
    auto update = [&](uint64_t* ma, uint32_t at, const uint64_t (&vv)[NV]) {
        if constexpr (CP) spec::apply_all<0, ACCS...>(ma, (uint32_t)GR, at, vv);
        else dev_::shared_row_update<NV>(ma, GR, (int)at, d, vv);
    };
    const int64_t nu = *n_units;
    for (int64_t u = blockIdx.x; u < nu; u += gridDim.x) {
        const part_unit un = units[u];
        // Replicas of this unit: every one for a piece of a split (large)
        // partition, where a few groups take most rows; otherwise one per 16
        // rows of a group, since each replica also costs set-up and merge
        // work (e.g. a 4K-row unit of ~256 groups keeps one).
        int R = reps;
        if (!un.split) {
            const int64_t q = (un.end - un.begin) / (16 * (int64_t)gpp);
            R = 1;
            while (R < reps && 2 * (int64_t)R <= q) R *= 2;
        }
        const uint32_t GRu = gcap * (uint32_t)R;  // words in use per accumulator
        const int rep = (int)(threadIdx.x & (unsigned)(R - 1));
        unsigned* my_counts = counts + rep;
        uint64_t* my_acc = acc + rep;
        for (uint32_t i = threadIdx.x; i < s_slots; i += HGB_NT) t.slots[i] = UD_EMPTY;
        if (KW == 8)
            for (uint32_t i = threadIdx.x; i < gcap; i += HGB_NT) t.gkey[i] = (kt)UD_UNSET;
        for (uint32_t i = threadIdx.x; i < GRu; i += HGB_NT) counts[i] = 0;
        for (int a = 0; a < NA; ++a) {
            const uint64_t idv = dev_::acc_ident(d.acc_op[a], d.acc_kind[a]);
            uint64_t* base = acc + (size_t)a * GR;
            for (uint32_t i = threadIdx.x; i < GRu; i += HGB_NT) base[i] = idv;
        }
        if (threadIdx.x == 0) { s_fill = 0; s_spill = 0; }
        __syncthreads();
        const int64_t tile = (int64_t)HGB_NT * HU_UNROLL;
        auto drain = [&](uint32_t off, bool live) {
            const int64_t i = un.begin + off;
            kt kq = 0;
            uint64_t vq[NV];
            if (live) {
                kq = (kt)ud_load_key<KW>(keys, i, key_kind);
                load_vals(i, vq);
            }
            const uint32_t hq = live ? key_hash<KW>(kq) : 0u;
            const uint32_t gq = d_find_or_insert_warp<KW>(t, live, kq, tag_of(kq, hq), hq >> shift);
            __syncwarp();
            if (!live) return;
            if (gq < gcap) {
                atomicAdd(&my_counts[gq * R], 1u);
                update(my_acc, gq * R, vq);
            } else {
                if (!s_spill) s_spill = 1;
                uint64_t* r = g_find_or_insert<KW>(g, d, kq, hq);
                if (r) g_update(r, d, vq, 1ull);
            }
        };
        int qfill = 0;
        for (int64_t base = un.begin; base < un.end; base += tile) {
            kt kw[HU_UNROLL];
            uint64_t v[HU_UNROLL][NV];
#pragma unroll
            for (int q = 0; q < HU_UNROLL; ++q) {
                const int64_t i = base + q * HGB_NT + threadIdx.x;
                if (i < un.end) {
                    kw[q] = (kt)ud_load_key<KW>(keys, i, key_kind);
                    load_vals(i, v[q]);
                }
            }
            // First probe of every row at once; a row whose home slot holds
            // another key (or a PENDING / spilled id) is queued for drain.
            uint32_t gid[HU_UNROLL];
#pragma unroll
            for (int q = 0; q < HU_UNROLL; ++q) {
                const bool valid = base + q * HGB_NT + threadIdx.x < un.end;
                gid[q] = 0xFFFFFFFFu;
                if (valid) {
                    const uint32_t h = key_hash<KW>(kw[q]);
                    const unsigned long long cur = ld_slot<KW>(&t.slots[(h >> shift) & t.mask]);
                    const uint32_t id = ud_id<KW>(cur);
                    if (ud_tag<KW>(cur) == tag_of(kw[q], h) && id < gcap &&
                        (KW == 4 || ((uint64_t)kw[q] != UD_UNSET &&
                                     (uint64_t)((volatile kt*)t.gkey)[id] == (uint64_t)kw[q])))
                        gid[q] = id;
                }
            }
#pragma unroll
            for (int q = 0; q < HU_UNROLL; ++q) {
                const int64_t i = base + q * HGB_NT + threadIdx.x;
                const bool valid = i < un.end;
                const bool hit = valid && gid[q] < gcap;
                const bool miss = valid && !hit;
                const unsigned mm = __ballot_sync(0xffffffffu, miss);
                if (miss) s_q[warp][qfill + __popc(mm & lt)] = (uint32_t)(i - un.begin);
                qfill += __popc(mm);
                if (hit) {
                    atomicAdd(&my_counts[gid[q] * R], 1u);
                    update(my_acc, gid[q] * R, v[q]);
                }
            }
            __syncwarp();
            while (qfill >= 32) {
                qfill -= 32;
                drain(s_q[warp][qfill + lane], true);
            }
        }
        drain(lane < qfill ? s_q[warp][lane] : 0u, lane < qfill);
        qfill = 0;
        __syncthreads();
        const uint32_t ng = min((uint32_t)s_fill, gcap);
        const bool final_groups = !un.split && !s_spill;
        if (final_groups) {
            if (threadIdx.x == 0) {
                s_base = atomicAdd(out_count, (unsigned long long)ng);
                if ((int64_t)(s_base + ng) > rec_cap) atomicExch(rec_ovf, 1);
            }
            __syncthreads();
        }
        const bool append = final_groups && (int64_t)(s_base + ng) <= rec_cap;
        if (append || !final_groups) {
            // Ids are dense: group j of the unit is record s_base + j.
            for (uint32_t j = threadIdx.x; j < ng; j += HGB_NT) {
                const uint64_t kwv = (uint64_t)t.gkey[j];
                unsigned long long c = 0;
                int first = -1;
                for (int rp = 0; rp < R; ++rp) {
                    const unsigned cr = counts[(size_t)j * R + rp];
                    c += cr;
                    if (cr && first < 0) first = rp;
                }
                uint64_t* r;
                if (append) {
                    r = out_recs + (s_base + j) * d.rec_words;
                    r[0] = kwv;
                    if (d.has_count) r[d.count_word] = c;
                } else {
                    if (first < 0) continue;
                    r = g_find_or_insert<KW>(g, d, kwv, key_hash<KW>(kwv));
                    if (!r) continue;
                    if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), c);
                }
                for (int a = 0; a < NA; ++a) {
                    uint64_t x = dev_::acc_ident(d.acc_op[a], d.acc_kind[a]);
                    if (first >= 0) {
                        x = acc[(size_t)a * GR + (size_t)j * R + first];
                        for (int rp = first + 1; rp < R; ++rp)
                            if (counts[(size_t)j * R + rp])
                                x = dev_::acc_combine(d.acc_op[a], d.acc_kind[a], x,
                                                      acc[(size_t)a * GR + (size_t)j * R + rp]);
                    }
                    if (append) r[d.acc_word0 + a] = x;
                    else dev_::acc_atomic(r + d.acc_word0 + a, d.acc_op[a], d.acc_kind[a], x);
                }
            }
        }
        __syncthreads();
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

// Shared-table geometry: S slots (load <= 1/2) and R accumulator replicas
// within a 200 KB budget (one 1024-thread CTA per SM).
int hash_smem_slots(const agg_desc& d, int key_width, int64_t groups_bound, int* replicas) {
    const size_t budget = 200 * 1024;
    const size_t per_rep = 4 + 8 * (size_t)d.n_acc;  // per slot per replica
    uint32_t s = 1u << 16;
    while (s > 64 && s * (key_width + per_rep) > budget) s >>= 1;
    if (groups_bound > 0 && groups_bound < (int64_t)s / 2) {
        uint32_t want = (uint32_t)next_pow2((uint64_t)groups_bound * 2);
        if (want < 64) want = 64;
        if (want < s) s = want;
    }
    size_t r = (budget - (size_t)s * key_width) / ((size_t)s * per_rep);
    if (r < 1) r = 1;
    if (r > 32) r = 32;
    // A power of two: with replicas innermost, lanes then spread evenly over
    // the banks.
    while (r & (r - 1)) r &= r - 1;
    *replicas = (int)r;
    return (int)s;
}

template <int KW, bool SMEM, int NV>
static void launch_hash_nv(int grid, size_t smem, cudaStream_t s, const void* keys, int64_t n, int kind,
                           const agg_desc& d, const gtable& g, uint32_t slots, int reps) {
    if (SMEM)
        GX_CUDA(cudaFuncSetAttribute(k_hash_groupby<KW, SMEM, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    k_hash_groupby<KW, SMEM, NV><<<grid, HGB_NT, smem, s>>>(keys, n, kind, d, g, SMEM ? slots : 0, SMEM ? reps : 1);
}

// Specialised instantiations: (op, kind, column) lists over 8-byte value columns.
template <class... ACCS>
static bool plan_matches(const agg_desc& d) {
    constexpr int ops[] = {ACCS::op...}, kinds[] = {ACCS::kind...}, cols[] = {ACCS::col...};
    if (d.n_acc != (int)sizeof...(ACCS)) return false;
    for (int c = 0; c < d.n_cols; ++c)
        if (d.col_width[c] != 8) return false;
    for (int a = 0; a < d.n_acc; ++a)
        if (d.acc_op[a] != ops[a] || d.acc_kind[a] != kinds[a] || d.acc_col[a] != cols[a]) return false;
    return true;
}

template <int KW, int NV, class... ACCS>
static bool try_spec(int grid, size_t smem, cudaStream_t s, const void* keys, int64_t n, int kind, const agg_desc& d,
                     const gtable& g, uint32_t slots, int reps) {
    if (d.n_cols != NV || !plan_matches<ACCS...>(d)) return false;
    GX_CUDA(cudaFuncSetAttribute(k_hash_groupby<KW, true, NV, ACCS...>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    k_hash_groupby<KW, true, NV, ACCS...><<<grid, HGB_NT, smem, s>>>(keys, n, kind, d, g, slots, reps);
    return true;
}

template <int KW>
static bool launch_spec(int grid, size_t smem, cudaStream_t s, const void* keys, int64_t n, int kind,
                        const agg_desc& d, const gtable& g, uint32_t slots, int reps) {
    using namespace spec;
    // SUM(int) [+ COUNT]
    if (try_spec<KW, 1, A<OP_SUM, VK_I, 0>>(grid, smem, s, keys, n, kind, d, g, slots, reps)) return true;
    // SUM(double)
    if (try_spec<KW, 1, A<OP_SUM, VK_F, 0>>(grid, smem, s, keys, n, kind, d, g, slots, reps)) return true;
    // SUM / MIN / MAX over an int64 and a float64 column [+ COUNT]
    if (try_spec<KW, 2, A<OP_SUM, VK_I, 0>, A<OP_MIN, VK_I, 0>, A<OP_MAX, VK_I, 0>, A<OP_SUM, VK_F, 1>,
                 A<OP_MIN, VK_F, 1>, A<OP_MAX, VK_F, 1>>(grid, smem, s, keys, n, kind, d, g, slots, reps))
        return true;
    // SUM over two int64 columns
    if (try_spec<KW, 2, A<OP_SUM, VK_I, 0>, A<OP_SUM, VK_I, 1>>(grid, smem, s, keys, n, kind, d, g, slots, reps))
        return true;
    return false;
}

template <int KW>
static void launch_hash(bool smem_mode, int nv, int grid, size_t smem, cudaStream_t s, const void* keys, int64_t n,
                        int kind, const agg_desc& d, const gtable& g, uint32_t slots, int reps) {
    if (smem_mode && !getenv("GX_HASH_GENERIC") && launch_spec<KW>(grid, smem, s, keys, n, kind, d, g, slots, reps))
        return;
#define GX_HL(SM, NV) \
    if (smem_mode == SM && nv == NV) return launch_hash_nv<KW, SM, NV>(grid, smem, s, keys, n, kind, d, g, slots, reps);
    GX_HL(true, 1) GX_HL(true, 2) GX_HL(true, 4) GX_HL(true, 8)
    GX_HL(false, 1) GX_HL(false, 2) GX_HL(false, 4) GX_HL(false, 8)
#undef GX_HL
}

// ---- partitioned units ----------------------------------------------------
struct units_args {
    const void* keys;
    int kind;
    const part_unit* units;
    const int64_t* n_units;
    uint32_t slots;
    int reps, shift;
    gtable g;
    uint64_t* orec;
    unsigned long long* ocount;
    int64_t rec_cap;
    int* rec_ovf;
};

template <int KW, int NV, class... ACCS>
static void launch_units(int grid, size_t smem, cudaStream_t s, const agg_desc& d, const units_args& a) {
    GX_CUDA(cudaFuncSetAttribute(k_hash_units<KW, NV, ACCS...>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    k_hash_units<KW, NV, ACCS...><<<grid, HGB_NT, smem, s>>>(a.keys, a.kind, d, a.units, a.n_units, a.slots, a.reps,
                                                             a.shift, a.g, a.orec, a.ocount, a.rec_cap, a.rec_ovf);
}

template <int KW, int NV, class... ACCS>
static bool try_units_spec(int grid, size_t smem, cudaStream_t s, const agg_desc& d, const units_args& a) {
    if (d.n_cols != NV || !plan_matches<ACCS...>(d)) return false;
    launch_units<KW, NV, ACCS...>(grid, smem, s, d, a);
    return true;
}

template <int KW, int NV, class... ACCS>
static bool launch_units_dense(int grid, size_t smem, cudaStream_t s, const agg_desc& d, const units_args& a,
                               uint32_t gcap, uint32_t gpp) {
    GX_PROF("partition_aggregate", s);
    GX_CUDA(cudaFuncSetAttribute(k_units_dense<KW, NV, ACCS...>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    k_units_dense<KW, NV, ACCS...><<<grid, HGB_NT, smem, s>>>(a.keys, a.kind, d, a.units, a.n_units, a.slots, gcap,
                                                              a.reps, gpp, a.shift, a.g, a.orec, a.ocount,
                                                              a.rec_cap, a.rec_ovf);
    return true;
}

template <int KW, int NV, class... ACCS>
static bool try_units_dense(int grid, size_t smem, cudaStream_t s, const agg_desc& d, const units_args& a,
                            uint32_t gcap, uint32_t gpp) {
    if (d.n_cols != NV || !plan_matches<ACCS...>(d)) return false;
    return launch_units_dense<KW, NV, ACCS...>(grid, smem, s, d, a, gcap, gpp);
}

// The dense-id kernel: a compiled plan when one matches (GX_HASH_GENERIC
// skips them), else the run-time aggregation list; false for more than four
// value columns.
template <int KW>
static bool units_dense_dispatch(int grid, size_t smem, cudaStream_t s, const agg_desc& d, const units_args& a,
                                 uint32_t gcap, uint32_t gpp) {
    using namespace spec;
    if (!getenv("GX_HASH_GENERIC")) {
        if (try_units_dense<KW, 1, A<OP_SUM, VK_I, 0>>(grid, smem, s, d, a, gcap, gpp)) return true;
        if (try_units_dense<KW, 1, A<OP_SUM, VK_F, 0>>(grid, smem, s, d, a, gcap, gpp)) return true;
        if (try_units_dense<KW, 2, A<OP_SUM, VK_I, 0>, A<OP_MIN, VK_I, 0>, A<OP_MAX, VK_I, 0>, A<OP_SUM, VK_F, 1>,
                            A<OP_MIN, VK_F, 1>, A<OP_MAX, VK_F, 1>>(grid, smem, s, d, a, gcap, gpp))
            return true;
        if (try_units_dense<KW, 2, A<OP_SUM, VK_I, 0>, A<OP_SUM, VK_I, 1>>(grid, smem, s, d, a, gcap, gpp)) return true;
    }
    if (d.n_cols > 4) return false;
    if (d.n_cols <= 1) return launch_units_dense<KW, 1>(grid, smem, s, d, a, gcap, gpp);
    if (d.n_cols <= 2) return launch_units_dense<KW, 2>(grid, smem, s, d, a, gcap, gpp);
    return launch_units_dense<KW, 4>(grid, smem, s, d, a, gcap, gpp);
}

template <int KW>
static void units_dispatch(int grid, size_t smem, cudaStream_t s, const agg_desc& d, const units_args& a) {
    using namespace spec;
    if (!getenv("GX_HASH_GENERIC")) {
        if (try_units_spec<KW, 1, A<OP_SUM, VK_I, 0>>(grid, smem, s, d, a)) return;
        if (try_units_spec<KW, 1, A<OP_SUM, VK_F, 0>>(grid, smem, s, d, a)) return;
        if (try_units_spec<KW, 2, A<OP_SUM, VK_I, 0>, A<OP_MIN, VK_I, 0>, A<OP_MAX, VK_I, 0>, A<OP_SUM, VK_F, 1>,
                           A<OP_MIN, VK_F, 1>, A<OP_MAX, VK_F, 1>>(grid, smem, s, d, a))
            return;
        if (try_units_spec<KW, 2, A<OP_SUM, VK_I, 0>, A<OP_SUM, VK_I, 1>>(grid, smem, s, d, a)) return;
    }
    const int nv = d.n_cols <= 1 ? 1 : d.n_cols <= 2 ? 2 : d.n_cols <= 4 ? 4 : 8;
    if (nv == 1) launch_units<KW, 1>(grid, smem, s, d, a);
    else if (nv == 2) launch_units<KW, 2>(grid, smem, s, d, a);
    else if (nv == 4) launch_units<KW, 4>(grid, smem, s, d, a);
    else launch_units<KW, 8>(grid, smem, s, d, a);
}

// Runs the hash group-by into a global table of `cap` records.
// Returns false when the table overflowed (caller retries larger).
// HASH through the dense-id unit kernel for a few thousand groups at most:
// the rows are cut into one range per SM, each a piece of one "partition"
// holding every group, aggregated in the CTA's dense table (group ids,
// replicated accumulators, no atomics on the global table per row) and
// merged into the global table once per range.
static bool hash_groupby_units(const col& key, const agg_desc& d, int64_t groups, const gtable& g, cudaStream_t s) {
    const int64_t n = key.n;
    const int ns = dev().sm_count;
    std::vector<part_unit> hu;
    const int64_t per = ceil_div(n, (int64_t)ns);
    for (int64_t b = 0; b < n; b += per) hu.push_back({b, std::min(n, b + per), 1, 0});
    const int64_t nu = (int64_t)hu.size();
    dbuf ub((size_t)nu * sizeof(part_unit) + 64, s);
    int64_t* d_nu = reinterpret_cast<int64_t*>(ub.get<char>() + (size_t)nu * sizeof(part_unit));
    GX_CUDA(cudaMemcpyAsync(ub.get(), hu.data(), (size_t)nu * sizeof(part_unit), cudaMemcpyHostToDevice, s));
    GX_CUDA(cudaMemcpyAsync(d_nu, &nu, 8, cudaMemcpyHostToDevice, s));
    // No unit is a whole partition, so no final records are appended.
    uint64_t* no_rec = reinterpret_cast<uint64_t*>(d_nu + 1);
    unsigned long long* no_cnt = reinterpret_cast<unsigned long long*>(d_nu + 2);
    int* no_ovf = reinterpret_cast<int*>(d_nu + 3);
    const bool ok = hash_units_aggregate(key.data, size_of(key.type), vkind_of(key.type), d, ub.get<part_unit>(), d_nu,
                                         groups, 0, g.recs, g.mask + 1, g.sentinel_flag, no_rec, no_cnt, 0, no_ovf, s,
                                         true);
    if (ok) GX_CUDA(cudaStreamSynchronize(s));  // the unit list lives in this scope
    return ok;
}

static bool hash_groupby_run(const col& key, int out_key_type, const agg_plan& p, uint64_t cap, int smem_mode,
                             int64_t units_groups, uint32_t s_slots, int reps, int64_t out_capacity, cudaStream_t s,
                             gx_table* out) {
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
    const bool units = key.n > 0 && units_groups > 0 && hash_groupby_units(key, d, units_groups, g, s);
    if (key.n > 0 && !units) {
        size_t smem = 0;
        if (smem_mode)
            smem = (((size_t)s_slots * kw + 15) & ~size_t(15)) + (((size_t)s_slots * 4 * reps + 15) & ~size_t(15)) +
                   (size_t)s_slots * reps * 8 * d.n_acc;
        int grid = grid_for(key.n, HGB_NT * HGB_UNROLL, smem_mode ? 1 : 2);
        GX_PROF("hash_groupby", s);
        int nv = d.n_cols <= 1 ? 1 : d.n_cols <= 2 ? 2 : d.n_cols <= 4 ? 4 : 8;
        if (kw == 4) launch_hash<4>(smem_mode, nv, grid, smem, s, key.data, key.n, kind, d, g, s_slots, reps);
        else launch_hash<8>(smem_mode, nv, grid, smem, s, key.data, key.n, kind, d, g, s_slots, reps);
        GX_LAUNCHED();
    }
    int hflags[2];
    GX_CUDA(cudaMemcpyAsync(hflags, flags.get(), sizeof(hflags), cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaStreamSynchronize(s));
    if (hflags[1]) return false;
    emit_groupby_output(p, recs.get<uint64_t>(), (int64_t)cap + 1, true, empty, (int64_t)cap,
                        flags.get<int>(), out_key_type, out_capacity, s, out);
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
    int reps = 1;
    uint32_t s_slots = (uint32_t)hash_smem_slots(p.d, size_of(key.type), bound_known ? bound : -1, &reps);
    // Shared tables only pay off when they can hold a useful share of the
    // keys (low cardinality, or skew that concentrates rows on few keys).
    bool smem_mode = bound <= (int64_t)s_slots * 8;
    if (!smem_mode && n > (1 << 16)) {
        // Many groups, but a skewed key column still pays for the shared
        // table: its heavy hitters stay there instead of serialising on one
        // global record (Zipf 1.0 over 2^16 keys: 16 ms instead of 192 ms at
        // 2^28 rows; uniform keys: 16.6 ms without, 21.7 ms with).  Switch it
        // on when the 8 most frequent keys of a 2^14-row sample carry >= 5%
        // of the sample.
        float f[GX_SEL_NUM_FEATURES];
        selector_features(key, f, s);
        float top = 0.f;
        for (int t = 0; t < 8; ++t) top += f[6 + t];
        smem_mode = top >= 0.05f;
    }
    if (const char* e = getenv("GX_HASH_SMEM")) smem_mode = atoi(e) != 0;
    // A few thousand groups at most: the dense-id unit kernel on row ranges.
    // (8-byte keys with a few hundred groups or fewer stay on the shared-table
    // kernel: int64 keys, G = 16: 2.16 ms there against 2.37 through units.)
    const int64_t units_groups = bound <= HASH_UNITS_MAX_GROUPS && (size_of(key.type) == 4 || bound > 256) &&
                                         smem_mode && !getenv("GX_HASH_NO_UNITS")
                                     ? bound
                                     : 0;
    int64_t out_cap = std::min<int64_t>(n, hint->groups_upper_bound > 0 ? hint->groups_upper_bound : n);
    for (int attempt = 0; attempt < 6; ++attempt) {
        if (hash_groupby_run(key, key_in.type, p, cap, smem_mode, units_groups, s_slots, reps, out_cap, s, out))
            return;
        cap *= 4;
    }
    fail(GX_EOVERFLOW, "hash group-by table overflow after retries");
}

bool hash_units_aggregate(const void* keys, int kw, int kind, const agg_desc& d, const part_unit* units,
                          const int64_t* n_units, int64_t gpp, int shift, uint64_t* grec, uint64_t gcap, int* gflags,
                          uint64_t* orec, unsigned long long* ocount, int64_t rec_cap, int* rec_ovf, cudaStream_t s,
                          bool dense_only) {
    const size_t budget = 200 * 1024;
    const size_t per_rep = 4 + 8 * (size_t)d.n_acc;
    // Slots for the fullest partition expected (Poisson tail), at load <= 1/4:
    // fewer rows miss their home slot, which beat accumulator replicas
    // (2048 slots × 1 replica: 3.03 ms for 7 aggregates at 2^28 rows, against
    // 1024 × 3 replicas: 3.26 ms).
    const double gmax = (double)gpp + 4.0 * std::sqrt((double)gpp) + 8.0;
    uint32_t slots = (uint32_t)next_pow2((uint64_t)std::max(64.0, 4.0 * gmax));
    const int grid = dev().sm_count;
    if (!getenv("GX_UNITS_SLOT_TABLE")) {
        // Dense group ids: slot words (8 B) at load <= 1/4, ids (and their
        // keys) for the fullest partition expected, and as many replicas (a
        // power of two, at most 16) as the budget holds.
        const uint32_t ids = (uint32_t)((((uint64_t)std::ceil(gmax)) + 31) & ~uint64_t(31));
        uint32_t dslots = slots;
        auto need = [&](size_t r) {
            return (size_t)dslots * 8 + (((size_t)ids * kw + 15) & ~size_t(15)) +
                   (((size_t)ids * r * 4 + 15) & ~size_t(15)) + (size_t)ids * r * 8 * d.n_acc;
        };
        // Slots at load <= 1/4, else <= 1/2 (e.g. ~2K groups with 7 aggregates).
        if (need(1) > budget) dslots = (uint32_t)next_pow2((uint64_t)std::max(64.0, 2.0 * gmax));
        size_t r = 16;
        while (r > 1 && need(r) > budget) r >>= 1;
        if (need(r) <= budget) {
            const units_args a{keys, kind, units, n_units, dslots, (int)r, shift,
                               gtable{grec, gcap - 1, gflags, gflags + 1}, orec, ocount, rec_cap, rec_ovf};
            const uint32_t g32 = (uint32_t)std::min<int64_t>(std::max<int64_t>(gpp, 1), ids);
            if (kw == 4 ? units_dense_dispatch<4>(grid, need(r), s, d, a, ids, g32)
                        : units_dense_dispatch<8>(grid, need(r), s, d, a, ids, g32)) {
                GX_LAUNCHED();
                return true;
            }
        }
    }
    if (dense_only) return false;
    // When load 1/4 does not fit (e.g. ~512 groups per partition with 7
    // aggregates), load 1/2 still beats the per-partition fallback kernel
    // by 3x (19.5 -> ~6.5 ms at 2^26.8 rows, 2^17 groups).
    if ((size_t)slots * (kw + per_rep) > budget) slots = (uint32_t)next_pow2((uint64_t)std::max(64.0, 2.0 * gmax));
    if ((size_t)slots * (kw + per_rep) > budget) return false;
    size_t reps = (budget - (size_t)slots * kw) / ((size_t)slots * per_rep);
    reps = std::max<size_t>(1, std::min<size_t>(32, reps));
    while (reps & (reps - 1)) reps &= reps - 1;
    const size_t smem = (((size_t)slots * kw + 15) & ~size_t(15)) + (((size_t)slots * 4 * reps + 15) & ~size_t(15)) +
                        (size_t)slots * reps * 8 * d.n_acc;
    units_args a{keys, kind, units, n_units, slots, (int)reps, shift,
                 gtable{grec, gcap - 1, gflags, gflags + 1}, orec, ocount, rec_cap, rec_ovf};
    GX_PROF("partition_aggregate", s);
    if (kw == 4) units_dispatch<4>(grid, smem, s, d, a);
    else units_dispatch<8>(grid, smem, s, d, a);
    GX_LAUNCHED();
    return true;
}

}  // namespace gx
