// gx_join_hash.cu — hash join and partitioned hash join (join_algo HASH and
// PARTITION).
//
// Replace the reference's hash-based inner equi-join plans:
//   * HASH: src/cuda/operators/join/hash_join.cu:22-145 builds a cuco
//     static_multiset of the build rows (src/cuda/containers/multiset.cuh:
//     112-278), counts every probe row's matches, then retrieves the pairs;
//   * PARTITION: src/cuda/operators/join/partition_hash_join.cu:26-697
//     radix-partitions both sides and joins each partition pair with a
//     chained hash table in shared memory.
// Both return every (build row, probe row) pair with equal keys — the same
// multiset as the sort plan; rows come out in probe order (HASH) or
// partition order (PARTITION), and build rows with equal keys in table
// order.
//
// B200 design:
//   * HASH: one open-addressing multiset of (key, build row) records at load
//     <= 1/2, built with one 64-bit compare-and-swap per row (4-byte keys
//     pack key and row in one record; 8-byte keys claim the row word and then
//     store the key), probed in 2048-row tiles: a count kernel sizes every
//     tile's output exactly, an exclusive scan places the tiles, and a write
//     kernel emits the pairs.  Each thread issues its eight rows' home-slot
//     loads together.  No atomics on the probe side, no output wrap.
//   * PARTITION: both sides are radix-partitioned (key + row id) by the hash
//     bits the PARTITION group-by uses, so that a build partition averages
//     ~1024 rows; one CTA per partition loads the build rows into a
//     shared-memory table (4096 slots; a larger partition, e.g. a hot key, is
//     taken 2048 rows at a time) and streams the probe partition through it,
//     counting first and writing second, the same exact-size scheme.
// Every walk ends: tables run at load <= 1/2, so an empty slot is always
// reached.
#include <algorithm>

#include "gx_join.h"

namespace gx {
namespace {

constexpr int HJ_NT = 256;
constexpr int HJ_IPT = 8;
constexpr int HJ_TILE = HJ_NT * HJ_IPT;
constexpr uint64_t HJ_EMPTY = ~0ull;

template <int KW>
__device__ __forceinline__ uint64_t hj_key(const void* keys, int64_t i, int kind) {
    if (KW == 4) return canon32(__ldg(static_cast<const unsigned*>(keys) + i), kind);
    return canon64(__ldg(static_cast<const unsigned long long*>(keys) + i), kind);
}
// The partition hash of the PARTITION group-by (fmix32 / folded fmix64).
template <int KW>
__device__ __forceinline__ uint32_t hj_hash(uint64_t k) {
    if (KW == 4) return fmix32((uint32_t)k);
    const uint64_t h = fmix64(k);
    return (uint32_t)(h ^ (h >> 32));
}

// Records: 4-byte keys: one word (build row << 32 | key); 8-byte keys: two
// words (build row, key).  An empty record has its row word all ones.
template <int KW>
__global__ void k_hj_build(const void* __restrict__ bkeys, int64_t nb, int kind, unsigned long long* __restrict__ table,
                           uint64_t mask) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nb; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = hj_key<KW>(bkeys, i, kind);
        uint64_t slot = hj_hash<KW>(k) & mask;
        if (KW == 4) {
            const unsigned long long rec = ((unsigned long long)i << 32) | (uint32_t)k;
            while (atomicCAS(table + slot, HJ_EMPTY, rec) != HJ_EMPTY) slot = (slot + 1) & mask;
        } else {
            while (atomicCAS(table + 2 * slot, HJ_EMPTY, (unsigned long long)i) != HJ_EMPTY) slot = (slot + 1) & mask;
            table[2 * slot + 1] = k;
        }
    }
}

// Walks the probe sequence of key k from `slot`; calls f(build_row) for
// every equal key.  Returns the number of matches.
template <int KW, class F>
__device__ __forceinline__ int hj_walk(const unsigned long long* __restrict__ table, uint64_t mask, uint64_t slot,
                                       uint64_t k, unsigned long long first, F&& f) {
    int c = 0;
    unsigned long long rec = first;
    for (;;) {
        if (KW == 4) {
            if (rec == HJ_EMPTY) break;
            if ((uint32_t)rec == (uint32_t)k) { f((int64_t)(rec >> 32)); ++c; }
        } else {
            if (rec == HJ_EMPTY) break;
            if (__ldg(table + 2 * slot + 1) == k) { f((int64_t)rec); ++c; }
        }
        slot = (slot + 1) & mask;
        rec = __ldg(table + (KW == 4 ? slot : 2 * slot));
    }
    return c;
}

// Count (WRITE = false: per-tile match totals) or write (WRITE = true: pairs
// at tile_off[tile] + the row-order prefix inside the tile).  Warp w of a
// block owns rows [tile + w*32*IPT, +32*IPT); row (k, lane) = k*32 + lane.
template <int KW, bool WRITE>
__global__ void __launch_bounds__(HJ_NT) k_hj_probe(const unsigned long long* __restrict__ table, uint64_t mask,
                                                     const void* __restrict__ pkeys, int64_t np, int kind,
                                                     int64_t* __restrict__ tile_cnt,
                                                     const int64_t* __restrict__ tile_off, join_out o) {
    __shared__ int64_t sm[HJ_NT / 32 + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row0 = blockIdx.x * (int64_t)HJ_TILE + warp * 32 * HJ_IPT + lane;
    uint64_t k[HJ_IPT], slot[HJ_IPT];
    unsigned long long first[HJ_IPT];
#pragma unroll
    for (int j = 0; j < HJ_IPT; ++j) {
        const int64_t i = row0 + j * 32;
        k[j] = i < np ? hj_key<KW>(pkeys, i, kind) : 0;
        slot[j] = hj_hash<KW>(k[j]) & mask;
    }
#pragma unroll
    for (int j = 0; j < HJ_IPT; ++j)
        first[j] = row0 + j * 32 < np ? __ldg(table + (KW == 4 ? slot[j] : 2 * slot[j])) : HJ_EMPTY;
    int cnt[HJ_IPT];
    int64_t mine = 0;
#pragma unroll
    for (int j = 0; j < HJ_IPT; ++j) {
        cnt[j] = hj_walk<KW>(table, mask, slot[j], k[j], first[j], [](int64_t) {});
        mine += cnt[j];
    }
    const int64_t wtot = dev_::warp_sum(mine);
    if constexpr (!WRITE) {
        if (lane == 0) sm[warp] = wtot;
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t t = 0;
            for (int w = 0; w < HJ_NT / 32; ++w) t += sm[w];
            tile_cnt[blockIdx.x] = t;
        }
    } else {
        int64_t total;
        int64_t wbase = dev_::block_exclusive_sum<HJ_NT, int64_t>(lane == 0 ? wtot : 0, sm, &total);
        wbase = __shfl_sync(0xffffffffu, wbase, 0) + tile_off[blockIdx.x];
        int64_t running = 0;
#pragma unroll
        for (int j = 0; j < HJ_IPT; ++j) {
            const int64_t inc = dev_::warp_inclusive_sum((int64_t)cnt[j]);
            int64_t pos = wbase + running + inc - cnt[j];
            running += __shfl_sync(0xffffffffu, inc, 31);
            const int64_t prow = row0 + j * 32;
            if (cnt[j])
                hj_walk<KW>(table, mask, slot[j], k[j], first[j],
                            [&](int64_t brow) { write_pair(o, pkeys, pos++, brow, prow); });
        }
    }
}

// ---------------------------------------------------------------------------
// Partitioned hash join: one CTA per partition pair (grid-stride).
// ---------------------------------------------------------------------------
constexpr int PJ_NT = 512;
constexpr int PJ_SLOTS = 4096;
constexpr int PJ_CHUNK = PJ_SLOTS / 2;
constexpr uint32_t PJ_EMPTY = 0xFFFFFFFFu;

struct pj_side {
    const void* keys;     // partitioned keys
    const int64_t* rows;  // original row id of each partitioned row
    const int64_t* start; // partition starts (P + 1)
};

template <int KW, bool WRITE>
__global__ void __launch_bounds__(PJ_NT) k_pj(pj_side b, pj_side p, int P, int R, int kind,
                                               const void* __restrict__ pkeys_orig, int64_t* __restrict__ part_cnt,
                                               const int64_t* __restrict__ part_off, join_out o) {
    using kt = typename std::conditional<KW == 4, uint32_t, unsigned long long>::type;
    extern __shared__ __align__(16) unsigned char pj_smem[];
    kt* skeys = reinterpret_cast<kt*>(pj_smem);
    uint32_t* srow = reinterpret_cast<uint32_t*>(pj_smem + (size_t)PJ_SLOTS * KW);  // chunk-local row, or empty
    __shared__ int64_t sm[PJ_NT / 32 + 1];
    const uint32_t mask = PJ_SLOTS - 1;
    for (int part = blockIdx.x; part < P; part += gridDim.x) {
        const int64_t bs = b.start[part], be = b.start[part + 1];
        const int64_t ps = p.start[part], pe = p.start[part + 1];
        int64_t base = WRITE ? part_off[part] : 0;
        int64_t count = 0;
        for (int64_t c0 = bs; c0 < be && ps < pe; c0 += PJ_CHUNK) {
            const int64_t c1 = min(be, c0 + PJ_CHUNK);
            for (int i = threadIdx.x; i < PJ_SLOTS; i += PJ_NT) srow[i] = PJ_EMPTY;
            __syncthreads();
            for (int64_t i = c0 + threadIdx.x; i < c1; i += PJ_NT) {
                const uint64_t k = hj_key<KW>(b.keys, i, kind);
                uint32_t slot = (hj_hash<KW>(k) >> R) & mask;
                while (atomicCAS(srow + slot, PJ_EMPTY, (uint32_t)(i - c0)) != PJ_EMPTY) slot = (slot + 1) & mask;
                skeys[slot] = (kt)k;
            }
            __syncthreads();
            for (int64_t q0 = ps; q0 < pe; q0 += PJ_NT) {
                const int64_t q = q0 + threadIdx.x;
                const bool live = q < pe;
                const uint64_t k = live ? hj_key<KW>(p.keys, q, kind) : 0;
                const uint32_t home = (hj_hash<KW>(k) >> R) & mask;
                int m = 0;
                if (live)
                    for (uint32_t s = home; srow[s] != PJ_EMPTY; s = (s + 1) & mask) m += skeys[s] == (kt)k;
                if constexpr (!WRITE) {
                    count += m;
                } else {
                    int64_t tot;
                    int64_t pos = base + dev_::block_exclusive_sum<PJ_NT, int64_t>((int64_t)m, sm, &tot);
                    base += tot;
                    if (m) {
                        const int64_t prow = p.rows[q];
                        for (uint32_t s = home; srow[s] != PJ_EMPTY; s = (s + 1) & mask)
                            if (skeys[s] == (kt)k) write_pair(o, pkeys_orig, pos++, b.rows[c0 + srow[s]], prow);
                    }
                }
            }
            __syncthreads();  // the table is rebuilt for the next chunk
        }
        if constexpr (!WRITE) {
            int64_t tot;
            dev_::block_exclusive_sum<PJ_NT, int64_t>(count, sm, &tot);
            if (threadIdx.x == 0) part_cnt[part] = tot;
        }
    }
}

struct sides {
    bool build_left;
    const col* bkey;
    const col* pkey;
};

sides pick_sides(const join_inputs& in) {
    require(in.lkey.type == in.rkey.type, "Join columns cannot have different types");
    const int kw = size_of(in.lkey.type);
    require(kw == 4 || kw == 8, "join: 4- or 8-byte key columns supported");
    require((int)in.lpay.size() <= MAX_PAY && (int)in.rpay.size() <= MAX_PAY, "join: too many payload columns");
    sides sd;
    sd.build_left = in.lkey.n <= in.rkey.n;
    sd.bkey = sd.build_left ? &in.lkey : &in.rkey;
    sd.pkey = sd.build_left ? &in.rkey : &in.lkey;
    return sd;
}

void check_max_out(const gx_join_hint& hint, int64_t total) {
    if (hint.max_out > 0 && total > hint.max_out)
        fail(GX_EOVERFLOW, "join output (" + std::to_string(total) + " rows) exceeds hint.max_out (" +
                               std::to_string(hint.max_out) + ")");
}

}  // namespace

void hash_join(const join_inputs& in, const gx_join_hint& hint, bool rowids_only, cudaStream_t s, gx_table* out) {
    const sides sd = pick_sides(in);
    const int kw = size_of(in.lkey.type), kind = vkind_of(in.lkey.type);
    const int64_t nb = sd.bkey->n, np = sd.pkey->n;
    require(nb < (int64_t)0x7FFFFFFF, "hash join: the build side (smaller input) must have fewer than 2^31 rows");
    const uint64_t cap = next_pow2((uint64_t)std::max<int64_t>(64, 2 * nb));
    const int64_t words = (int64_t)cap * (kw == 4 ? 1 : 2);
    dbuf table((size_t)words * 8, s);
    fill_u64(table.get(), HJ_EMPTY, words, s);
    if (nb > 0) {
        GX_PROF("join_build_hash", s);
        if (kw == 4) k_hj_build<4><<<grid_for(nb, 256, 8), 256, 0, s>>>(sd.bkey->data, nb, kind, table.get<unsigned long long>(), cap - 1);
        else k_hj_build<8><<<grid_for(nb, 256, 8), 256, 0, s>>>(sd.bkey->data, nb, kind, table.get<unsigned long long>(), cap - 1);
        GX_LAUNCHED();
    }
    const int64_t ntiles = ceil_div(std::max<int64_t>(np, 1), HJ_TILE);
    dbuf tc((size_t)ntiles * 8, s), toff((size_t)(ntiles + 1) * 8, s);
    int64_t total = 0;
    join_out none;
    std::memset(&none, 0, sizeof(none));
    if (np > 0 && nb > 0) {
        GX_PROF("join_probe_count", s);
        if (kw == 4) k_hj_probe<4, false><<<(unsigned)ntiles, HJ_NT, 0, s>>>(table.get<unsigned long long>(), cap - 1, sd.pkey->data, np, kind, tc.get<int64_t>(), nullptr, none);
        else k_hj_probe<8, false><<<(unsigned)ntiles, HJ_NT, 0, s>>>(table.get<unsigned long long>(), cap - 1, sd.pkey->data, np, kind, tc.get<int64_t>(), nullptr, none);
        GX_LAUNCHED();
        exclusive_scan_i64(tc.get<int64_t>(), toff.get<int64_t>(), ntiles, s);
        total = read_scalar(toff.get<int64_t>() + ntiles, s);
    }
    check_max_out(hint, total);
    join_out o = make_outputs(in, sd.build_left, rowids_only, false, true, total, s, out);
    if (total > 0) {
        GX_PROF("join_probe_write", s);
        if (kw == 4) k_hj_probe<4, true><<<(unsigned)ntiles, HJ_NT, 0, s>>>(table.get<unsigned long long>(), cap - 1, sd.pkey->data, np, kind, nullptr, toff.get<int64_t>(), o);
        else k_hj_probe<8, true><<<(unsigned)ntiles, HJ_NT, 0, s>>>(table.get<unsigned long long>(), cap - 1, sd.pkey->data, np, kind, nullptr, toff.get<int64_t>(), o);
        GX_LAUNCHED();
    }
    GX_CUDA(cudaStreamSynchronize(s));
}

void partition_hash_join(const join_inputs& in, const gx_join_hint& hint, bool rowids_only, cudaStream_t s,
                         gx_table* out) {
    const sides sd = pick_sides(in);
    const int kw = size_of(in.lkey.type), kind = vkind_of(in.lkey.type);
    const int64_t nb = sd.bkey->n, np = sd.pkey->n;
    int64_t total = 0;
    if (nb == 0 || np == 0) {
        make_outputs(in, sd.build_left, rowids_only, false, true, 0, s, out);
        return;
    }
    // About 1024 build rows per partition: a chunk of PJ_CHUNK rows covers
    // nearly every partition in one table build.
    const int R = std::max(1, std::min(16, ilog2_ceil((uint64_t)ceil_div(nb, 1024))));
    const int P = 1 << R;
    dbuf bk((size_t)nb * kw, s), br((size_t)nb * 8, s), bst((size_t)(P + 1) * 8, s);
    dbuf pk((size_t)np * kw, s), pr((size_t)np * 8, s), pst((size_t)(P + 1) * 8, s);
    hash_partition_rows(*sd.bkey, R, bk.get(), br.get<int64_t>(), bst.get<int64_t>(), s);
    hash_partition_rows(*sd.pkey, R, pk.get(), pr.get<int64_t>(), pst.get<int64_t>(), s);
    pj_side b{bk.get(), br.get<int64_t>(), bst.get<int64_t>()};
    pj_side p{pk.get(), pr.get<int64_t>(), pst.get<int64_t>()};
    const size_t smem = (size_t)PJ_SLOTS * (kw + 4);
    // 8-byte keys need 48 KB of dynamic shared memory, the default limit.
    static per_device_flag attr;
    attr.once([] {
        GX_CUDA(cudaFuncSetAttribute(k_pj<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, PJ_SLOTS * 12));
        GX_CUDA(cudaFuncSetAttribute(k_pj<8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, PJ_SLOTS * 12));
    });
    const int grid = std::min(P, dev().sm_count * 4);
    dbuf pc((size_t)P * 8, s), poff((size_t)(P + 1) * 8, s);
    join_out none;
    std::memset(&none, 0, sizeof(none));
    {
        GX_PROF("join_probe_count", s);
        if (kw == 4) k_pj<4, false><<<grid, PJ_NT, smem, s>>>(b, p, P, R, kind, sd.pkey->data, pc.get<int64_t>(), nullptr, none);
        else k_pj<8, false><<<grid, PJ_NT, smem, s>>>(b, p, P, R, kind, sd.pkey->data, pc.get<int64_t>(), nullptr, none);
        GX_LAUNCHED();
    }
    exclusive_scan_i64(pc.get<int64_t>(), poff.get<int64_t>(), P, s);
    total = read_scalar(poff.get<int64_t>() + P, s);
    check_max_out(hint, total);
    join_out o = make_outputs(in, sd.build_left, rowids_only, false, true, total, s, out);
    if (total > 0) {
        GX_PROF("join_probe_write", s);
        if (kw == 4) k_pj<4, true><<<grid, PJ_NT, smem, s>>>(b, p, P, R, kind, sd.pkey->data, nullptr, poff.get<int64_t>(), o);
        else k_pj<8, true><<<grid, PJ_NT, smem, s>>>(b, p, P, R, kind, sd.pkey->data, nullptr, poff.get<int64_t>(), o);
        GX_LAUNCHED();
    }
    GX_CUDA(cudaStreamSynchronize(s));
}

}  // namespace gx
