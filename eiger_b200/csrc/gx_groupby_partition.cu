// gx_groupby_partition.cu — partition-based group-by (PARTITION, PARTITION_GFUR).
//
// Replaces gamax::groupby::partition::groupby / groupby_gfur
// (src/cuda/operators/groupby/groupby_partition.cu:557-707).  Same shape as
// the reference — hash-partition the rows so each partition's groups fit a
// shared-memory table, then aggregate one partition per CTA — with three
// changes:
//   * partition id = fmix(key) on R radix bits (R chosen from the group
//     estimate, or hint.radix_bits) instead of a fixed 16; rows are moved by
//     one multi-column scatter per 8-bit digit (GFTR moves key + every value
//     column, GFUR key + row id) instead of one CUB sort per column;
//   * partitions larger than a threshold are split into work units so a
//     Zipf-hot partition is spread over many CTAs (the reference assigns one
//     CTA per partition, groupby_partition.cu:433);
//   * a partition whose distinct keys overflow its shared table spills to a
//     global table instead of throwing (groupby_partition.cu:543-549).
#include <algorithm>

#include "gx_groupby.h"

namespace gx {
namespace {

constexpr int PS_NT = 512;
constexpr int PS_WARPS = PS_NT / 32;
constexpr int PS_IPT = 8;
constexpr int PS_TILE = PS_NT * PS_IPT;
constexpr int PS_BINS = 256;

template <int KW>
__device__ __forceinline__ uint32_t part_hash(uint64_t kb) {
    if (KW == 4) return fmix32((uint32_t)kb);
    uint64_t h = fmix64(kb);
    return (uint32_t)(h ^ (h >> 32));
}
template <int KW>
__device__ __forceinline__ uint64_t ld_key(const void* p, int64_t i, int kind) {
    if (KW == 4) return canon32(__ldg(static_cast<const unsigned*>(p) + i), kind);
    return canon64(__ldg(static_cast<const unsigned long long*>(p) + i), kind);
}

struct move_cols {
    int n;
    const void* in[MAX_VCOLS + 2];
    void* out[MAX_VCOLS + 2];
    int width[MAX_VCOLS + 2];
    int iota[MAX_VCOLS + 2];  // 1: the column is the row id (input ignored)
};

// Stable multi-column scatter by one hash digit: ranks are computed once with
// a warp multisplit, then each column is staged through shared memory in
// digit order and written out in contiguous runs.
template <int KW>
__global__ void __launch_bounds__(PS_NT) k_part_scatter(const void* __restrict__ keys, int64_t n, int kind,
                                                         int shift, int dbits, int64_t ntiles,
                                                         const int64_t* __restrict__ offsets, move_cols mc) {
    __shared__ unsigned whist[PS_WARPS * PS_BINS];
    __shared__ int64_t gbase[PS_BINS];
    __shared__ unsigned dbase[PS_BINS];
    extern __shared__ __align__(16) unsigned long long part_dyn[];
    unsigned long long* stage = part_dyn;                                        // [PS_TILE]
    unsigned short* sdig = reinterpret_cast<unsigned short*>(part_dyn + PS_TILE);  // [PS_TILE]

    const int bins = 1 << dbits;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < PS_WARPS * PS_BINS; i += PS_NT) whist[i] = 0;
    __syncthreads();
    const int64_t tile_base = blockIdx.x * (int64_t)PS_TILE;
    const int tile_n = (int)min((int64_t)PS_TILE, n - tile_base);
    const unsigned lt = (1u << lane) - 1u;
    unsigned dig[PS_IPT], rank[PS_IPT];
#pragma unroll
    for (int k = 0; k < PS_IPT; ++k) {
        int local = warp * 32 * PS_IPT + k * 32 + lane;
        bool valid = local < tile_n;
        unsigned d = valid ? (part_hash<KW>(ld_key<KW>(keys, tile_base + local, kind)) >> shift) & (bins - 1) : 0xFFFFu;
        dig[k] = d;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned r = __popc(peers & lt);
        unsigned prior = valid ? whist[warp * PS_BINS + d] : 0;
        rank[k] = prior + r;
        __syncwarp();
        if (valid && r == 0) whist[warp * PS_BINS + d] = prior + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x < PS_BINS) {
        unsigned run = 0;
        if ((int)threadIdx.x < bins)
            for (int w = 0; w < PS_WARPS; ++w) {
                unsigned c = whist[w * PS_BINS + threadIdx.x];
                whist[w * PS_BINS + threadIdx.x] = run;
                run += c;
            }
        dbase[threadIdx.x] = run;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned v[PS_BINS / 32], s = 0;
#pragma unroll
        for (int j = 0; j < PS_BINS / 32; ++j) { v[j] = dbase[lane * (PS_BINS / 32) + j]; s += v[j]; }
        unsigned run = dev_::warp_inclusive_sum(s) - s;
#pragma unroll
        for (int j = 0; j < PS_BINS / 32; ++j) { dbase[lane * (PS_BINS / 32) + j] = run; run += v[j]; }
    }
    __syncthreads();
    if ((int)threadIdx.x < bins)
        gbase[threadIdx.x] = offsets[(int64_t)threadIdx.x * ntiles + blockIdx.x] - (int64_t)dbase[threadIdx.x];
    unsigned pos[PS_IPT];
#pragma unroll
    for (int k = 0; k < PS_IPT; ++k) {
        int local = warp * 32 * PS_IPT + k * 32 + lane;
        if (local < tile_n) {
            pos[k] = dbase[dig[k]] + whist[warp * PS_BINS + dig[k]] + rank[k];
            sdig[pos[k]] = (unsigned short)dig[k];
        }
    }
    __syncthreads();
    int64_t orow[PS_IPT];  // output row of each staged position this thread writes
#pragma unroll
    for (int m = 0; m < PS_IPT; ++m) {
        const int j = threadIdx.x + m * PS_NT;
        orow[m] = j < tile_n ? gbase[sdig[j]] + j : 0;
    }
    for (int c = 0; c < mc.n; ++c) {
        __syncthreads();
        const int w = mc.width[c];
#pragma unroll
        for (int k = 0; k < PS_IPT; ++k) {
            int local = warp * 32 * PS_IPT + k * 32 + lane;
            if (local < tile_n) {
                int64_t i = tile_base + local;
                unsigned long long x;
                if (mc.iota[c]) x = (unsigned long long)i;
                else if (w == 8) x = __ldg(static_cast<const unsigned long long*>(mc.in[c]) + i);
                else x = __ldg(static_cast<const unsigned*>(mc.in[c]) + i);
                stage[pos[k]] = x;
            }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < PS_IPT; ++m) {
            const int j = threadIdx.x + m * PS_NT;
            if (j >= tile_n) break;
            if (w == 8) static_cast<unsigned long long*>(mc.out[c])[orow[m]] = stage[j];
            else static_cast<unsigned*>(mc.out[c])[orow[m]] = (unsigned)stage[j];
        }
    }
}

// The same scatter for NC <= 3 columns with every column's values loaded into
// registers up front, so all of a tile's global loads are in flight together
// (the general kernel loads one column per staging round).
template <int KW, int NC>
__global__ void __launch_bounds__(PS_NT, 2) k_part_scatter_r(const void* __restrict__ keys, int64_t n, int kind,
                                                           int shift, int dbits, int64_t ntiles,
                                                           const int64_t* __restrict__ offsets, move_cols mc) {
    __shared__ unsigned whist[PS_WARPS * PS_BINS];
    __shared__ int64_t gbase[PS_BINS];
    __shared__ unsigned dbase[PS_BINS];
    extern __shared__ __align__(16) unsigned long long part_dyn[];
    unsigned long long* stage = part_dyn;                                          // [PS_TILE]
    unsigned short* sdig = reinterpret_cast<unsigned short*>(part_dyn + PS_TILE);  // [PS_TILE]

    const int bins = 1 << dbits;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < PS_WARPS * PS_BINS; i += PS_NT) whist[i] = 0;
    const int64_t tile_base = blockIdx.x * (int64_t)PS_TILE;
    const int tile_n = (int)min((int64_t)PS_TILE, n - tile_base);
    unsigned long long x[NC][PS_IPT];
#pragma unroll
    for (int k = 0; k < PS_IPT; ++k) {
        const int local = warp * 32 * PS_IPT + k * 32 + lane;
        const int64_t i = tile_base + local;
        const bool valid = local < tile_n;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            x[c][k] = 0;
            if (valid) {
                if (mc.iota[c]) x[c][k] = (unsigned long long)i;
                else if (mc.width[c] == 8) x[c][k] = __ldg(static_cast<const unsigned long long*>(mc.in[c]) + i);
                else x[c][k] = __ldg(static_cast<const unsigned*>(mc.in[c]) + i);
            }
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    unsigned dig[PS_IPT], rank[PS_IPT];
#pragma unroll
    for (int k = 0; k < PS_IPT; ++k) {
        const int local = warp * 32 * PS_IPT + k * 32 + lane;
        const bool valid = local < tile_n;
        uint64_t kb;
        if (KW == 4) kb = canon32((uint32_t)x[0][k], kind);
        else kb = canon64(x[0][k], kind);
        const unsigned d = valid ? (part_hash<KW>(kb) >> shift) & (bins - 1) : 0xFFFFu;
        dig[k] = d;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned r = __popc(peers & lt);
        const unsigned prior = valid ? whist[warp * PS_BINS + d] : 0;
        rank[k] = prior + r;
        __syncwarp();
        if (valid && r == 0) whist[warp * PS_BINS + d] = prior + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x < PS_BINS) {
        unsigned run = 0;
        if ((int)threadIdx.x < bins)
            for (int w = 0; w < PS_WARPS; ++w) {
                const unsigned c = whist[w * PS_BINS + threadIdx.x];
                whist[w * PS_BINS + threadIdx.x] = run;
                run += c;
            }
        dbase[threadIdx.x] = run;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned v[PS_BINS / 32], s = 0;
#pragma unroll
        for (int j = 0; j < PS_BINS / 32; ++j) { v[j] = dbase[lane * (PS_BINS / 32) + j]; s += v[j]; }
        unsigned run = dev_::warp_inclusive_sum(s) - s;
#pragma unroll
        for (int j = 0; j < PS_BINS / 32; ++j) { dbase[lane * (PS_BINS / 32) + j] = run; run += v[j]; }
    }
    __syncthreads();
    if ((int)threadIdx.x < bins)
        gbase[threadIdx.x] = offsets[(int64_t)threadIdx.x * ntiles + blockIdx.x] - (int64_t)dbase[threadIdx.x];
    unsigned pos[PS_IPT];
#pragma unroll
    for (int k = 0; k < PS_IPT; ++k) {
        const int local = warp * 32 * PS_IPT + k * 32 + lane;
        if (local < tile_n) {
            pos[k] = dbase[dig[k]] + whist[warp * PS_BINS + dig[k]] + rank[k];
            sdig[pos[k]] = (unsigned short)dig[k];
        }
    }
    // Output row of each staged position this thread writes, computed once
    // for all columns.
    __syncthreads();
    int64_t orow[PS_IPT];
#pragma unroll
    for (int m = 0; m < PS_IPT; ++m) {
        const int j = threadIdx.x + m * PS_NT;
        orow[m] = j < tile_n ? gbase[sdig[j]] + j : 0;
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PS_IPT; ++k) {
            const int local = warp * 32 * PS_IPT + k * 32 + lane;
            if (local < tile_n) stage[pos[k]] = x[c][k];
        }
        __syncthreads();
        const int w = mc.width[c];
#pragma unroll
        for (int m = 0; m < PS_IPT; ++m) {
            const int j = threadIdx.x + m * PS_NT;
            if (j >= tile_n) break;
            if (w == 8) static_cast<unsigned long long*>(mc.out[c])[orow[m]] = stage[j];
            else static_cast<unsigned*>(mc.out[c])[orow[m]] = (unsigned)stage[j];
        }
    }
}

// ---------------------------------------------------------------------------
// Bulk-copy scatter: one persistent CTA per SM walks its tiles (blockIdx.x,
// + gridDim.x, ...), with each tile's column slices brought into shared
// memory by the copy engine (cp.async.bulk on an mbarrier) one tile ahead, so
// the loads of tile t+1 overlap the ranking and writes of tile t and no
// column value occupies a register.  STABLE ranks a tile as k_part_scatter
// does (digit, then row order); otherwise each row's rank within its digit
// is one shared atomic (any order inside a (digit, tile) run).  Each output
// position j then reads its source row from the shared copy and writes every
// column to gbase[digit] + j.  Used when every loaded column starts on a
// 16-byte boundary and two tiles of the columns fit in shared memory.
// ---------------------------------------------------------------------------
constexpr int PB_NT = 1024;
constexpr int PB_WARPS = PB_NT / 32;
constexpr int PB_IPT = PS_TILE / PB_NT;  // 4
constexpr uint32_t PB_WAIT_LIMIT = 1u << 22;

struct pb_layout {
    uint32_t in_off[MAX_VCOLS + 2];  // column c's slice within one stage
    uint32_t stage_bytes;            // one tile of every loaded column
    uint32_t whist, qsum, pk, gbase, dbase, total;
};

// Shared-memory layout; the per-warp counts of the stable ranking are only
// laid out when `stable`.
__host__ __device__ inline pb_layout pb_make_layout(const move_cols& mc, bool stable) {
    pb_layout L{};
    uint32_t o = 0;
    for (int c = 0; c < mc.n; ++c) {
        L.in_off[c] = o;
        if (!mc.iota[c]) o += (uint32_t)PS_TILE * (uint32_t)mc.width[c];
    }
    L.stage_bytes = o;
    o *= 2;
    L.whist = o; if (stable) o += PB_WARPS * PS_BINS * 2;   // u16 per-warp digit counts
    L.qsum = o;  if (stable) o += 4 * PS_BINS * 2;          // u16 sums over 8-warp quarters
    L.pk = o;    o += PS_TILE * 4;              // u32 per staged position: source row | digit << 16
    L.gbase = o; o += PS_BINS * 8;              // int64 output base per digit
    L.dbase = o; o += PS_BINS * 4;              // u32 first staged position per digit
    L.total = o;
    return L;
}

// IMG: the digit is bits [shift, shift + dbits) of the key's order-preserving
// image (a stable LSD radix-sort pass, `ip`); otherwise of the key's
// partition hash (`kind`).
template <int KW, int NC, bool STABLE, bool IMG>
__global__ void __launch_bounds__(PB_NT, 1) k_part_scatter_bulk(const void* __restrict__ keys, int64_t n, int kind,
                                                                img_params ip, int shift, int dbits, int64_t ntiles,
                                                                const int64_t* __restrict__ offsets, move_cols mc,
                                                                pb_layout L, int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char pb_smem[];
    __shared__ __align__(8) unsigned long long bars[2];
    __shared__ unsigned wsum[PS_BINS / 32];
    __shared__ unsigned thist[PS_BINS];  // unstable ranking: running count per digit
    __shared__ int s_err;
    unsigned short* whist = reinterpret_cast<unsigned short*>(pb_smem + L.whist);
    unsigned short* qsum = reinterpret_cast<unsigned short*>(pb_smem + L.qsum);
    unsigned* pk = reinterpret_cast<unsigned*>(pb_smem + L.pk);
    int64_t* gbase = reinterpret_cast<int64_t*>(pb_smem + L.gbase);
    unsigned* dbase = reinterpret_cast<unsigned*>(pb_smem + L.dbase);

    const int bins = 1 << dbits;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const uint32_t bar0 = dev_::smem_addr(&bars[0]);
    // Issues the copies of tile `tile` into stage `b` (thread 0 only; full
    // tiles only — the last, partial tile is loaded with plain loads).
    auto issue = [&](int64_t tile, int b) {
        const uint32_t bar = bar0 + 8u * (uint32_t)b;
        dev_::mbar_arrive_expect_tx(bar, L.stage_bytes);
        const uint32_t base = dev_::smem_addr(pb_smem) + (uint32_t)b * L.stage_bytes;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (mc.iota[c]) continue;
            const uint32_t bytes = (uint32_t)PS_TILE * (uint32_t)mc.width[c];
            dev_::bulk_load_g2s(base + L.in_off[c],
                                static_cast<const unsigned char*>(mc.in[c]) + tile * (int64_t)bytes, bytes, bar);
        }
    };
    auto full = [&](int64_t tile) { return (tile + 1) * (int64_t)PS_TILE <= n; };
    unsigned char* stage = nullptr;
    // Digit of the tile's row `local` (key column of the current stage).
    auto digit_at = [&](int local) -> unsigned {
        uint64_t kb;
        if (KW == 4) kb = reinterpret_cast<const unsigned*>(stage + L.in_off[0])[local];
        else kb = reinterpret_cast<const unsigned long long*>(stage + L.in_off[0])[local];
        if constexpr (IMG) return (unsigned)((key_image<KW>(kb, ip) >> shift) & (uint64_t)(bins - 1));
        kb = KW == 4 ? canon32((uint32_t)kb, kind) : canon64(kb, kind);
        return (part_hash<KW>(kb) >> shift) & (bins - 1);
    };
    if (t == 0) {
        dev_::mbar_init(bar0, 1);
        dev_::mbar_init(bar0 + 8, 1);
        dev_::mbar_init_fence();
        s_err = 0;
    }
    if (t < PS_BINS) thist[t] = 0;
    __syncthreads();
    // A copy into stage b was issued and not yet waited for: tracked by
    // thread 0, the only issuer.
    // Bit b of `pending` / `phase`: stage b's copy state and barrier parity.
    uint32_t pending = 0, phase = 0;
    if (t == 0) {
        for (int b = 0; b < 2; ++b) {
            const int64_t tile = blockIdx.x + (int64_t)b * gridDim.x;
            if (tile < ntiles && full(tile)) { issue(tile, b); pending |= 1u << b; }
        }
    }
    const unsigned lt = (1u << lane) - 1u;
    int it = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int b = it & 1;
        stage = pb_smem + (size_t)b * L.stage_bytes;
        const int64_t tile_base = tile * (int64_t)PS_TILE;
        const int tile_n = (int)min((int64_t)PS_TILE, n - tile_base);
        // Digit offsets of this tile (read early; used after the scan).
        const int64_t my_off = t < bins ? offsets[(int64_t)t * ntiles + tile] : 0;
        if (full(tile)) {
            if (dev_::mbar_wait_bounded(bar0 + 8u * (uint32_t)b, (phase >> b) & 1u, PB_WAIT_LIMIT)) {
                phase ^= 1u << b;
                pending &= ~(1u << b);
            } else {
                s_err = 1;
            }
        } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (mc.iota[c]) continue;
                if (mc.width[c] == 8) {
                    auto* d = reinterpret_cast<unsigned long long*>(stage + L.in_off[c]);
                    for (int i = t; i < tile_n; i += PB_NT)
                        d[i] = __ldg(static_cast<const unsigned long long*>(mc.in[c]) + tile_base + i);
                } else {
                    auto* d = reinterpret_cast<unsigned*>(stage + L.in_off[c]);
                    for (int i = t; i < tile_n; i += PB_NT)
                        d[i] = __ldg(static_cast<const unsigned*>(mc.in[c]) + tile_base + i);
                }
            }
            __syncthreads();
        }
        // Rank the tile's rows within their digit.  STABLE (every pass after
        // the first of a multi-pass partition, which LSD order needs): per-warp
        // counts over rows warp*128 + k*32 + lane, then a cross-warp prefix.
        // Otherwise one shared atomic per row gives an arbitrary order within
        // each (digit, tile) run, which a single-pass partition allows.
        unsigned dig[PB_IPT], rank[PB_IPT];
        unsigned tot = 0, incl = 0;
        if constexpr (STABLE) {
            for (int i = lane; i < PS_BINS; i += 32) whist[warp * PS_BINS + i] = 0;
            __syncwarp();
#pragma unroll
            for (int k = 0; k < PB_IPT; ++k) {
                const int local = warp * 32 * PB_IPT + k * 32 + lane;
                const bool valid = local < tile_n;
                const unsigned d = valid ? digit_at(local) : 0xFFFFu;
                dig[k] = d;
                const unsigned peers = __match_any_sync(0xffffffffu, d);
                const unsigned r = __popc(peers & lt);
                const unsigned prior = valid ? whist[warp * PS_BINS + d] : 0;
                rank[k] = prior + r;
                __syncwarp();
                if (valid && r == 0) whist[warp * PS_BINS + d] = (unsigned short)(prior + __popc(peers));
                __syncwarp();
            }
            __syncthreads();
            if (s_err) break;
            // Cross-warp exclusive prefix per digit: thread (q, bin) sums warps 8q..8q+7.
            const int bq = t & (PS_BINS - 1), q = t >> 8;
            unsigned v[8], s = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) { v[j] = whist[(q * 8 + j) * PS_BINS + bq]; s += v[j]; }
            qsum[q * PS_BINS + bq] = (unsigned short)s;
            __syncthreads();
            unsigned run = 0;
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                const unsigned x = qsum[qq * PS_BINS + bq];
                if (qq < q) run += x;
                tot += x;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) { whist[(q * 8 + j) * PS_BINS + bq] = (unsigned short)run; run += v[j]; }
        } else {
#pragma unroll
            for (int k = 0; k < PB_IPT; ++k) {
                const int local = warp * 32 * PB_IPT + k * 32 + lane;
                const bool valid = local < tile_n;
                dig[k] = valid ? digit_at(local) : 0u;
                rank[k] = valid ? atomicAdd(&thist[dig[k]], 1u) : 0u;
            }
            __syncthreads();
            if (s_err) break;
            if (t < PS_BINS) {
                tot = thist[t];
                thist[t] = 0;  // ready for the next tile
            }
        }
        if (t < PS_BINS) {
            incl = dev_::warp_inclusive_sum(tot);
            if (lane == 31) wsum[warp] = incl;
        }
        __syncthreads();
        if (t < PS_BINS) {
            unsigned ex = incl - tot;
            for (int w = 0; w < warp; ++w) ex += wsum[w];
            dbase[t] = ex;
            gbase[t] = my_off - (int64_t)ex;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PB_IPT; ++k) {
            const int local = warp * 32 * PB_IPT + k * 32 + lane;
            if (local < tile_n) {
                const unsigned pos = dbase[dig[k]] + (STABLE ? (unsigned)whist[warp * PS_BINS + dig[k]] : 0u) + rank[k];
                pk[pos] = (unsigned)local | (dig[k] << 16);
            }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < PB_IPT; ++m) {
            const int j = t + m * PB_NT;
            if (j >= tile_n) break;
            const unsigned e = pk[j];
            const int64_t orow = gbase[e >> 16] + j;
            const int sr = (int)(e & 0xFFFFu);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (mc.iota[c]) {
                    static_cast<unsigned long long*>(mc.out[c])[orow] = (unsigned long long)(tile_base + sr);
                } else if (mc.width[c] == 8) {
                    static_cast<unsigned long long*>(mc.out[c])[orow] =
                        reinterpret_cast<const unsigned long long*>(stage + L.in_off[c])[sr];
                } else {
                    static_cast<unsigned*>(mc.out[c])[orow] = reinterpret_cast<const unsigned*>(stage + L.in_off[c])[sr];
                }
            }
        }
        __syncthreads();
        // Stage b is free again: prefetch the tile after next into it (the
        // proxy fence orders this CTA's reads of the stage before the copy).
        if (t == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const int64_t nt = tile + 2 * (int64_t)gridDim.x;
            if (nt < ntiles && full(nt)) { issue(nt, b); pending |= 1u << b; }
        }
    }
    if (s_err) {
        // A copy never completed: report it and wait (bounded) for the copies
        // still in flight into this CTA's shared memory before leaving.
        if (t == 0) {
            atomicExch(err, 1);
            for (int b = 0; b < 2; ++b)
                if ((pending >> b) & 1u) dev_::mbar_wait_bounded(bar0 + 8u * (uint32_t)b, (phase >> b) & 1u, PB_WAIT_LIMIT);
        }
        __syncthreads();
    }
}

// Per-tile digit counts with one warp per 4096-row tile: a warp-private
// shared histogram, no block-wide barriers, 16 loads in flight per thread.
constexpr int PH_NT = 256;
constexpr int PH_WARPS = PH_NT / 32;
template <int KW>
__global__ void __launch_bounds__(PH_NT) k_part_hist(const void* __restrict__ keys, int64_t n, int kind, int shift,
                                                       int dbits, int64_t ntiles, int64_t* __restrict__ counts) {
    __shared__ unsigned hist[PH_WARPS][PS_BINS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned bmask = (1u << dbits) - 1u;
    unsigned* h = hist[warp];
    for (int i = lane; i < PS_BINS; i += 32) h[i] = 0;
    __syncwarp();
    const bool vec = (reinterpret_cast<uintptr_t>(keys) & 15) == 0;
    for (int64_t tile = blockIdx.x * (int64_t)PH_WARPS + warp; tile < ntiles; tile += (int64_t)gridDim.x * PH_WARPS) {
        const int64_t base = tile * (int64_t)PS_TILE;
        const int tile_n = (int)min((int64_t)PS_TILE, n - base);
        if (vec && tile_n == PS_TILE) {
            // Full tile from a 16-byte aligned column: 16-byte loads, eight
            // in flight per thread (32 keys of 4 bytes, or 16 of 8).
            constexpr int KPV = 16 / KW, NVEC = PS_TILE / KPV, B = 8;
            const uint4* kv = reinterpret_cast<const uint4*>(static_cast<const unsigned char*>(keys) + base * KW);
            for (int j0 = 0; j0 < NVEC; j0 += 32 * B) {
                uint4 x[B];
#pragma unroll
                for (int q = 0; q < B; ++q) x[q] = __ldcs(kv + j0 + q * 32 + lane);
#pragma unroll
                for (int q = 0; q < B; ++q) {
                    if (KW == 4) {
                        const unsigned w[4] = {x[q].x, x[q].y, x[q].z, x[q].w};
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                            atomicAdd(&h[(part_hash<4>(canon32(w[e], kind)) >> shift) & bmask], 1u);
                    } else {
                        const uint64_t w[2] = {((uint64_t)x[q].y << 32) | x[q].x, ((uint64_t)x[q].w << 32) | x[q].z};
#pragma unroll
                        for (int e = 0; e < 2; ++e)
                            atomicAdd(&h[(part_hash<8>(canon64(w[e], kind)) >> shift) & bmask], 1u);
                    }
                }
            }
            __syncwarp();
            for (int i = lane; i <= (int)bmask; i += 32) {
                counts[(int64_t)i * ntiles + tile] = h[i];
                h[i] = 0;
            }
            __syncwarp();
            continue;
        }
        constexpr int B = 16;
        for (int j0 = 0; j0 < PS_TILE; j0 += 32 * B) {
            uint64_t kb[B];
#pragma unroll
            for (int q = 0; q < B; ++q) {
                const int local = j0 + q * 32 + lane;
                kb[q] = local < tile_n ? ld_key<KW>(keys, base + local, kind) : 0;
            }
#pragma unroll
            for (int q = 0; q < B; ++q) {
                const int local = j0 + q * 32 + lane;
                if (local < tile_n) atomicAdd(&h[(part_hash<KW>(kb[q]) >> shift) & bmask], 1u);
            }
        }
        __syncwarp();
        for (int i = lane; i <= (int)bmask; i += 32) {
            counts[(int64_t)i * ntiles + tile] = h[i];
            h[i] = 0;
        }
        __syncwarp();
    }
}

__global__ void k_starts_from_offsets(const int64_t* __restrict__ offs, int64_t ntiles, int P, int64_t n,
                                      int64_t* __restrict__ ps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < P) ps[p] = offs[(int64_t)p * ntiles];
    else if (p == P) ps[P] = n;
}

// Work units: partition p split into ceil(size/T) units.
__global__ void k_unit_counts(const int64_t* __restrict__ part_start, int P, int64_t T,
                              int64_t* __restrict__ ucount) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < P) {
        int64_t sz = part_start[p + 1] - part_start[p];
        ucount[p] = sz == 0 ? 0 : (sz + T - 1) / T;
    }
}
using unit = part_unit;
__global__ void k_unit_fill(const int64_t* __restrict__ part_start, const int64_t* __restrict__ uoff, int P,
                            int64_t T, unit* __restrict__ units) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    int64_t b = part_start[p], e = part_start[p + 1];
    int64_t u0 = uoff[p], nu = uoff[p + 1] - u0;
    for (int64_t u = 0; u < nu; ++u) {
        unit x;
        x.begin = b + u * T;
        x.end = min(e, x.begin + T);
        x.split = nu > 1;
        x.pad = 0;
        units[u0 + u] = x;
    }
}

constexpr uint64_t PG_EMPTY4 = ~0ull;
constexpr uint64_t PG_EMPTY8 = 0x8000000000000000ull;
constexpr int PA_NT = 512;

struct pglobal {
    uint64_t* recs;  // (cap + 1) records, the last one for the key equal to the empty marker
    uint64_t mask;
    int* sentinel_flag;
    int* overflow;
};

template <int KW>
__device__ __forceinline__ uint64_t* pg_find(const pglobal& t, const agg_desc& d, uint64_t kw, uint32_t h) {
    const uint64_t EMPTY = KW == 4 ? PG_EMPTY4 : PG_EMPTY8;
    if (KW == 8 && kw == EMPTY) {
        atomicExch(t.sentinel_flag, 1);
        return t.recs + (t.mask + 1) * d.rec_words;
    }
    uint64_t slot = (h * 0x9E3779B1u) & t.mask;
    for (uint64_t p = 0, lim = t.mask < GX_PROBE_LIMIT ? t.mask : GX_PROBE_LIMIT - 1; p <= lim; ++p) {
        uint64_t* r = t.recs + slot * d.rec_words;
        uint64_t cur = *(volatile uint64_t*)r;
        if (cur == kw) return r;
        if (cur == EMPTY) {
            unsigned long long old = atomicCAS((unsigned long long*)r, (unsigned long long)EMPTY, (unsigned long long)kw);
            if (old == EMPTY || old == kw) return r;
        }
        slot = (slot + 1) & t.mask;
    }
    atomicExch(t.overflow, 1);
    return nullptr;
}

// One CTA per work unit (grid-stride over units).  Shared table layout:
// keys[S] (u64) | counts[S] (u32) | acc[A][S] (u64).
template <int KW>
__global__ void __launch_bounds__(PA_NT) k_part_agg(const void* __restrict__ pkeys,
                                                     const int64_t* __restrict__ prow,  // GFUR row ids (or null)
                                                     move_cols pvals,                  // GFTR partitioned values
                                                     int kind, agg_desc d, const unit* __restrict__ units,
                                                     const int64_t* __restrict__ n_units, uint32_t S, int rbits,
                                                     pglobal g, uint64_t* __restrict__ out_recs,
                                                     unsigned long long* __restrict__ out_count, int64_t rec_cap,
                                                     int* __restrict__ rec_overflow) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_fill;
    __shared__ int s_spilled;
    __shared__ unsigned long long s_base;
    unsigned long long* skeys = reinterpret_cast<unsigned long long*>(smem);
    unsigned* scnt = reinterpret_cast<unsigned*>(smem + (size_t)S * 8);
    uint64_t* sacc = reinterpret_cast<uint64_t*>(smem + (size_t)S * 12);
    const uint64_t EMPTY = KW == 4 ? PG_EMPTY4 : PG_EMPTY8;
    const uint32_t mask = S - 1;
    const int limit = (int)(S - S / 4);
    const int64_t nu = *n_units;
    for (int64_t u = blockIdx.x; u < nu; u += gridDim.x) {
        const unit un = units[u];
        for (uint32_t i = threadIdx.x; i < S; i += PA_NT) { skeys[i] = EMPTY; scnt[i] = 0; }
        for (int a = 0; a < d.n_acc; ++a) {
            int op = d.acc_op[a], kd = d.acc_kind[a];
            uint64_t idv = op == OP_MIN ? (kd == VK_I ? 0x7FFFFFFFFFFFFFFFull : (kd == VK_U ? ~0ull : 0x7FF0000000000000ull))
                         : op == OP_MAX ? (kd == VK_I ? 0x8000000000000000ull : (kd == VK_U ? 0ull : 0xFFF0000000000000ull))
                         : 0ull;
            for (uint32_t i = threadIdx.x; i < S; i += PA_NT) sacc[(size_t)a * S + i] = idv;
        }
        if (threadIdx.x == 0) { s_fill = 0; s_spilled = 0; }
        __syncthreads();
        for (int64_t i = un.begin + threadIdx.x; i < un.end; i += PA_NT) {
            uint64_t kw = ld_key<KW>(pkeys, i, kind);
            uint32_t h = part_hash<KW>(kw);
            uint64_t v[MAX_VCOLS];
            if (prow) {
                int64_t src = prow[i];
#pragma unroll
                for (int c = 0; c < MAX_VCOLS; ++c)
                    if (c < d.n_cols) v[c] = dev_::load_lane(d.col_ptr[c], d.col_width[c], d.col_kind[c], src);
            } else {
#pragma unroll
                for (int c = 0; c < MAX_VCOLS; ++c)
                    if (c < d.n_cols) v[c] = dev_::load_lane(pvals.out[c], d.col_width[c], d.col_kind[c], i);
            }
            // Slot from the hash bits above the partition bits.
            uint32_t slot = (h >> rbits) & mask;
            int found = -1;
            if (!(KW == 8 && kw == EMPTY)) {
                for (uint32_t p = 0; p <= mask; ++p) {
                    unsigned long long cur = ((volatile unsigned long long*)skeys)[slot];
                    if (cur == kw) { found = (int)slot; break; }
                    if (cur == EMPTY) {
                        if (*(volatile int*)&s_fill >= limit) break;
                        unsigned long long old = atomicCAS(&skeys[slot], (unsigned long long)EMPTY, (unsigned long long)kw);
                        if (old == EMPTY) { atomicAdd(&s_fill, 1); found = (int)slot; break; }
                        if (old == kw) { found = (int)slot; break; }
                    }
                    slot = (slot + 1) & mask;
                }
            }
            if (found >= 0) {
                if (d.has_count) atomicAdd(&scnt[found], 1u);
                dev_::shared_row_update<MAX_VCOLS>(sacc, S, found, d, v);
            } else {
                if (!s_spilled) s_spilled = 1;
                uint64_t* r = pg_find<KW>(g, d, kw, h);
                if (r) {
                    if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), 1ull);
                    for (int a = 0; a < d.n_acc; ++a)
                        dev_::acc_atomic(r + d.acc_word0 + a, d.acc_op[a], d.acc_kind[a], dev_::pick(v, d.acc_col[a]));
                }
            }
        }
        __syncthreads();
        // A unit that spilled may hold a key both here and in the spill table
        // (a row raced the table closing), so it merges like a split unit.
        if (!un.split && !s_spilled) {
            // Whole partition in this CTA: its groups are final; append them densely.
            if (threadIdx.x == 0) {
                s_base = atomicAdd(out_count, (unsigned long long)s_fill);
                if ((int64_t)(s_base + s_fill) > rec_cap) atomicExch(rec_overflow, 1);
            }
            __syncthreads();
            if ((int64_t)(s_base + s_fill) > rec_cap) { __syncthreads(); continue; }
            // Compact occupied slots in slot order with a block scan.
            __shared__ int64_t scan_sm[PA_NT / 32 + 1];
            int64_t running = 0;
            for (uint32_t i0 = 0; i0 < S; i0 += PA_NT) {
                uint32_t i = i0 + threadIdx.x;
                bool live = i < S && skeys[i] != EMPTY;
                int64_t tot;
                int64_t ex = dev_::block_exclusive_sum<PA_NT, int64_t>(live ? 1 : 0, scan_sm, &tot);
                if (live) {
                    uint64_t* r = out_recs + (s_base + running + ex) * d.rec_words;
                    r[0] = skeys[i];
                    if (d.has_count) r[d.count_word] = scnt[i];
                    for (int a = 0; a < d.n_acc; ++a) r[d.acc_word0 + a] = sacc[(size_t)a * S + i];
                }
                running += tot;
            }
        } else {
            for (uint32_t i = threadIdx.x; i < S; i += PA_NT) {
                unsigned long long k = skeys[i];
                if (k == EMPTY) continue;
                uint64_t* r = pg_find<KW>(g, d, k, part_hash<KW>(k));
                if (!r) continue;
                if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), (unsigned long long)scnt[i]);
                for (int a = 0; a < d.n_acc; ++a)
                    dev_::acc_atomic(r + d.acc_word0 + a, d.acc_op[a], d.acc_kind[a], sacc[(size_t)a * S + i]);
            }
        }
        __syncthreads();
    }
}

// Append the occupied records of the global spill table after the dense ones.
__global__ void k_append_global(const uint64_t* __restrict__ g, int64_t cap, int rec_words, uint64_t empty,
                                const int* __restrict__ sentinel_flag, uint64_t* __restrict__ out,
                                unsigned long long* __restrict__ out_count, int64_t rec_cap,
                                int* __restrict__ rec_overflow) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= cap; r += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t* src = g + r * rec_words;
        bool live = r < cap ? src[0] != empty : *sentinel_flag != 0;
        if (!live) continue;
        unsigned long long pos = atomicAdd(out_count, 1ull);
        if ((int64_t)pos >= rec_cap) { atomicExch(rec_overflow, 1); continue; }
        for (int w = 0; w < rec_words; ++w) out[pos * rec_words + w] = src[w];
    }
}

}  // namespace

void partition_starts(const void* keys, int kw, int64_t n, int kind, int R, int64_t* ps, cudaStream_t s);

namespace {

// The bulk-copy scatter applies to 1..4 moved columns when every loaded
// column is 4 or 8 bytes wide and 16-byte aligned, and two tiles of them fit
// in shared memory (four columns: up to 24 B per row, single-pass ranking).
static bool bulk_scatter_ok(const move_cols& mc, const pb_layout& L) {
    if (mc.n < 1 || mc.n > 4) return false;
    for (int c = 0; c < mc.n; ++c) {
        if (mc.iota[c]) continue;
        if (mc.width[c] != 4 && mc.width[c] != 8) return false;
        if (reinterpret_cast<uintptr_t>(mc.in[c]) % 16 != 0) return false;
    }
    return L.total <= (uint32_t)dev().max_smem_optin - 2048;
}

template <int KW>
void part_pass(const void* kin, int64_t n, int kind, int shift, int dbits, move_cols& mc, int64_t* counts,
               int64_t* offs, int* err, bool stable, cudaStream_t s) {
    int64_t ntiles = ceil_div(n, PS_TILE);
    const int hist_grid = (int)std::min<int64_t>(ceil_div(ntiles, PH_WARPS), (int64_t)dev().sm_count * 8);
    k_part_hist<KW><<<hist_grid, PH_NT, 0, s>>>(kin, n, kind, shift, dbits, ntiles, counts);
    GX_LAUNCHED();
    exclusive_scan_i64(counts, offs, ((int64_t)1 << dbits) * ntiles, s);
    const pb_layout L = pb_make_layout(mc, stable);
    if (mc.n >= 2 && !getenv("GX_PART_NO_BULK") && bulk_scatter_ok(mc, L)) {
        static per_device_flag battr;
        battr.once([] {
            const int lim = dev().max_smem_optin - 2048;
            GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<KW, 2, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
            GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<KW, 3, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
            GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<KW, 2, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
            GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<KW, 3, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
            GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<KW, 4, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
            GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<KW, 4, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        });
        const int grid = (int)std::min<int64_t>(ntiles, dev().sm_count);
        const img_params no_img{};
        GX_PROF("partition_scatter", s);
#define GX_PB_LAUNCH(NCV, ST)                                                                                       \
    k_part_scatter_bulk<KW, NCV, ST, false><<<grid, PB_NT, L.total, s>>>(kin, n, kind, no_img, shift, dbits, ntiles, \
                                                                          offs, mc, L, err)
        if (mc.n == 2 && stable) GX_PB_LAUNCH(2, true);
        else if (mc.n == 2) GX_PB_LAUNCH(2, false);
        else if (mc.n == 3 && stable) GX_PB_LAUNCH(3, true);
        else if (mc.n == 3) GX_PB_LAUNCH(3, false);
        else if (stable) GX_PB_LAUNCH(4, true);
        else GX_PB_LAUNCH(4, false);
#undef GX_PB_LAUNCH
        GX_LAUNCHED();
        return;
    }
    const int dyn = PS_TILE * 10;
    static per_device_flag attr;
    attr.once([dyn] {
        GX_CUDA(cudaFuncSetAttribute(k_part_scatter<KW>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
        GX_CUDA(cudaFuncSetAttribute(k_part_scatter_r<KW, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
        GX_CUDA(cudaFuncSetAttribute(k_part_scatter_r<KW, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    });
    GX_PROF("partition_scatter", s);
    if (mc.n == 2) k_part_scatter_r<KW, 2><<<(unsigned)ntiles, PS_NT, dyn, s>>>(kin, n, kind, shift, dbits, ntiles, offs, mc);
    else if (mc.n == 3) k_part_scatter_r<KW, 3><<<(unsigned)ntiles, PS_NT, dyn, s>>>(kin, n, kind, shift, dbits, ntiles, offs, mc);
    else k_part_scatter<KW><<<(unsigned)ntiles, PS_NT, dyn, s>>>(kin, n, kind, shift, dbits, ntiles, offs, mc);
    GX_LAUNCHED();
}

}  // namespace

void partition_groupby(const col& key_in, const agg_plan& p, gx_groupby_hint* hint, bool gfur, cudaStream_t s,
                       gx_table* out) {
    owned_col widened;
    col key = key_in;
    if (size_of(key.type) < 4) {
        widened = widen_to_32(key, s);
        key.data = widened.buf.get();
        key.type = widened.type;
    }
    const int64_t n = key.n;
    const int kw = size_of(key.type);
    const int kind = vkind_of(key.type);
    const agg_desc& d = p.d;
    // Shared table of one partition: small on purpose.  Random shared-memory
    // atomics on B200 cost roughly one pass per distinct 128-byte segment a
    // warp touches, so a partition's table is sized for its expected groups
    // (a few hundred bytes per accumulator) rather than for the whole SM:
    // the radix bits are chosen so each partition holds about 16 groups.
    size_t per_slot = 8 + 4 + 8 * (size_t)d.n_acc;
    uint32_t S_max = 1u << 14;
    while (S_max > 256 && S_max * per_slot > 200 * 1024) S_max >>= 1;
    int64_t bound = std::min<int64_t>(n, hint->groups_upper_bound > 0 ? hint->groups_upper_bound : n);
    if (!(hint->groups_upper_bound > 0 && hint->groups_upper_bound < n) && n > (1 << 16))
        bound = std::min<int64_t>(n, ndv_estimate(key, s) * 9 / 8 + 64);
    // About 256 groups per partition: a shared table of ~1K slots holds them
    // (with a few accumulator replicas), and up to 2^16 groups need a single
    // 8-bit radix pass.
    int64_t gpp = gfur ? 16 : 256;
    for (int c = 0; c < d.n_cols; ++c)
        if (d.col_width[c] < 4) gpp = 16;
    if (const char* e = getenv("GX_PART_GROUPS")) gpp = std::max<int64_t>(1, atoll(e));
    int R = hint->radix_bits;
    if (R <= 0) R = ilog2_ceil((uint64_t)std::max<int64_t>(1, ceil_div(bound, gpp)));
    R = std::max(1, std::min(16, R));
    hint->radix_bits = R;
    const int P = 1 << R;
    // Four slots per expected group absorbs the spread of groups across partitions.
    uint32_t S = (uint32_t)std::min<uint64_t>(S_max, std::max<uint64_t>(64, next_pow2((uint64_t)ceil_div(bound, P) * 4)));

    // Partitioned copies.
    move_cols mc;
    std::memset(&mc, 0, sizeof(mc));
    // Partitioned copies (scratch slots 0..8 and, for a second pass, 9..17).
    std::vector<void*> bufs_a, bufs_b;
    auto add_col = [&](const void* in, int w, int iota) {
        int c = mc.n++;
        mc.in[c] = in;
        mc.width[c] = w;
        mc.iota[c] = iota;
        bufs_a.push_back(thread_scratch((int)bufs_a.size(), (size_t)std::max<int64_t>(n, 1) * w));
        mc.out[c] = bufs_a.back();
    };
    // 1- and 2-byte value columns are read through row ids (GFUR) instead of
    // being moved by the 4/8-byte scatter.
    for (int c = 0; c < d.n_cols; ++c) gfur = gfur || d.col_width[c] < 4;
    add_col(key.data, kw, 0);
    if (gfur) add_col(nullptr, 8, 1);
    else
        for (int c = 0; c < d.n_cols; ++c) add_col(d.col_ptr[c], d.col_width[c], 0);

    int64_t ntiles = ceil_div(std::max<int64_t>(n, 1), PS_TILE);
    int64_t* counts = static_cast<int64_t*>(thread_scratch(SCRATCH_SLOTS - 2, (size_t)PS_BINS * ntiles * 8));
    int64_t* offs = static_cast<int64_t*>(thread_scratch(SCRATCH_SLOTS - 1, (size_t)PS_BINS * ntiles * 8 + 8));
    // Unit offsets [0, P] then one word the bulk-copy scatter sets when a
    // copy wait gave up, so one read after the unit setup fetches both.
    dbuf uoff((size_t)(P + 2) * 8, s);
    int* perr = reinterpret_cast<int*>(uoff.get<int64_t>() + P + 1);
    GX_CUDA(cudaMemsetAsync(perr, 0, 8, s));
    int passes = (R + 7) / 8;
    // Two digit passes ping-pong between bufs_a and bufs_b.
    if (passes == 2)
        for (int c = 0; c < mc.n; ++c)
            bufs_b.push_back(thread_scratch(MAX_VCOLS + 1 + c, (size_t)std::max<int64_t>(n, 1) * mc.width[c]));
    if (n > 0) {
        int shift = 0;
        for (int ps = 0; ps < passes; ++ps) {
            int dbits = std::min(8, R - shift);
            move_cols m = mc;
            if (passes == 2 && ps == 0) {
                for (int c = 0; c < mc.n; ++c) m.out[c] = bufs_b[c];
            } else if (passes == 2 && ps == 1) {
                for (int c = 0; c < mc.n; ++c) { m.in[c] = bufs_b[c]; m.iota[c] = 0; m.out[c] = bufs_a[c]; }
            }
            const void* kin = m.in[0];
            // Only the first digit pass may leave rows unordered within a run.
            const bool stable = ps > 0;
            if (kw == 4) part_pass<4>(kin, n, kind, shift, dbits, m, counts, offs, perr, stable, s);
            else part_pass<8>(kin, n, kind, shift, dbits, m, counts, offs, perr, stable, s);
            shift += dbits;
        }
    }
    // Partition starts: the keys are now grouped by partition id, so
    // part_start[p] is the first row whose id is >= p.
    dbuf pstart((size_t)(P + 1) * 8, s);
    if (passes == 1 && n > 0) {
        // One pass: the scanned digit counts already hold each partition's
        // start (bin p's offset in the first tile).
        k_starts_from_offsets<<<(unsigned)ceil_div(P + 1, 256), 256, 0, s>>>(offs, ntiles, P, n,
                                                                            pstart.get<int64_t>());
        GX_LAUNCHED();
    } else {
        partition_starts(mc.out[0], kw, n, kind, R, pstart.get<int64_t>(), s);
    }

    // Work units.
    // Split threshold: partitions above twice the mean size are split (Zipf
    // hot partitions), and with few partitions every partition is split so
    // that about four units per SM exist.
    int64_t T = std::max<int64_t>(1 << 14, std::min<int64_t>(2 * ceil_div(n, P), ceil_div(n, (int64_t)dev().sm_count * 8)));
    dbuf ucount((size_t)P * 8, s);
    k_unit_counts<<<(unsigned)ceil_div(P, 256), 256, 0, s>>>(pstart.get<int64_t>(), P, T, ucount.get<int64_t>());
    GX_LAUNCHED();
    exclusive_scan_i64(ucount.get<int64_t>(), uoff.get<int64_t>(), P, s);
    int64_t max_units = P + ceil_div(n, T) + 1;
    dbuf units((size_t)max_units * sizeof(unit), s);
    k_unit_fill<<<(unsigned)ceil_div(P, 256), 256, 0, s>>>(pstart.get<int64_t>(), uoff.get<int64_t>(), P, T,
                                                           units.get<unit>());
    GX_LAUNCHED();

    uint64_t empty = kw == 4 ? PG_EMPTY4 : PG_EMPTY8;
    // Split units merge through the spill table, so size it for every group
    // when any partition was split; otherwise it only catches overflow.  When
    // a table for every group is small (<= 64 MB) it is used either way, so
    // the host does not wait for the unit count before the aggregation; the
    // scatter's timeout flag is then read with the final flags.
    int64_t tail[2] = {0, 0};
    const int64_t live_parts = std::min<int64_t>(P, n);
    const uint64_t all_groups = std::max<uint64_t>(1u << 16, next_pow2((uint64_t)bound * 2));
    uint64_t gcap = 1u << 16;
    const bool tail_later = (all_groups + 1) * (uint64_t)d.rec_words * 8 <= (64ull << 20);
    if (tail_later) {
        gcap = all_groups;
    } else {
        GX_CUDA(cudaMemcpyAsync(tail, uoff.get<int64_t>() + P, sizeof(tail), cudaMemcpyDeviceToHost, s));
        GX_CUDA(cudaStreamSynchronize(s));
        if ((int)tail[1]) fail(GX_ETIMEOUT, "partition scatter: a bulk copy into shared memory did not complete");
        // Also when partitions hold more groups than a shared table (radix
        // bits forced low by the hint): their overflow spills here.
        if (tail[0] > live_parts || ceil_div(bound, (int64_t)P) > 512) gcap = all_groups;
    }
    int64_t out_cap = std::min<int64_t>(n, hint->groups_upper_bound > 0 ? hint->groups_upper_bound : n);
    // Output records: sized from the group bound, grown (up to n) on overflow.
    int64_t rec_cap = std::max<int64_t>(1, std::min<int64_t>(n, std::max<int64_t>(bound + bound / 4, 4096)));
    for (int attempt = 0; attempt < 8; ++attempt) {
        dbuf grec((gcap + 1) * d.rec_words * 8, s);
        dbuf flags(32, s);  // [0] sentinel, [1] spill overflow, [8..15] count, [16] record overflow
        GX_CUDA(cudaMemsetAsync(flags.get(), 0, 32, s));
        init_records(grec.get<uint64_t>(), (int64_t)gcap + 1, d, empty, s);
        uint64_t* orec = static_cast<uint64_t*>(thread_scratch(SCRATCH_SLOTS - 3, (size_t)rec_cap * d.rec_words * 8));
        unsigned long long* ocount = reinterpret_cast<unsigned long long*>(flags.get<char>() + 8);
        int* rec_ovf = reinterpret_cast<int*>(flags.get<char>() + 16);
        pglobal g{grec.get<uint64_t>(), gcap - 1, flags.get<int>(), flags.get<int>() + 1};
        bool done_units = false;
        if (n > 0 && !gfur && !getenv("GX_PART_OLD_AGG")) {
            // Rows were moved with their values: aggregate with the shared
            // hash-table kernel over the partitioned copies.
            agg_desc pd = d;
            for (int c = 0; c < d.n_cols; ++c) pd.col_ptr[c] = mc.out[c + 1];
            done_units = hash_units_aggregate(mc.out[0], kw, kind, pd, units.get<part_unit>(), uoff.get<int64_t>() + P,
                                              ceil_div(bound, (int64_t)P), R, grec.get<uint64_t>(), gcap,
                                              flags.get<int>(), orec, ocount, rec_cap, rec_ovf, s);
        }
        if (n > 0 && !done_units) {
            size_t smem = (size_t)S * per_slot;
            int per_sm = (int)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / std::max<size_t>(smem, 1)));
            int grid = dev().sm_count * per_sm;
            move_cols pv;
            std::memset(&pv, 0, sizeof(pv));
            if (!gfur)
                for (int c = 0; c + 1 < mc.n; ++c) pv.out[c] = mc.out[c + 1];
            const int64_t* prow = gfur ? static_cast<const int64_t*>(mc.out[1]) : nullptr;
            GX_PROF("partition_aggregate", s);
            if (kw == 4) {
                GX_CUDA(cudaFuncSetAttribute(k_part_agg<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                k_part_agg<4><<<grid, PA_NT, smem, s>>>(mc.out[0], prow, pv, kind, d, units.get<unit>(),
                                                       uoff.get<int64_t>() + P, S, R, g, orec, ocount,
                                                       rec_cap, rec_ovf);
            } else {
                GX_CUDA(cudaFuncSetAttribute(k_part_agg<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                k_part_agg<8><<<grid, PA_NT, smem, s>>>(mc.out[0], prow, pv, kind, d, units.get<unit>(),
                                                       uoff.get<int64_t>() + P, S, R, g, orec, ocount,
                                                       rec_cap, rec_ovf);
            }
            GX_LAUNCHED();
        }
        // The spill records are appended before the overflow flags are read,
        // so one read decides: a spill-table overflow discards this attempt.
        k_append_global<<<grid_for((int64_t)gcap + 1, 256, 4), 256, 0, s>>>(grec.get<uint64_t>(), (int64_t)gcap,
                                                                          d.rec_words, empty, flags.get<int>(),
                                                                          orec, ocount, rec_cap,
                                                                          rec_ovf);
        GX_LAUNCHED();
        int fl[8];
        GX_CUDA(cudaMemcpyAsync(fl, flags.get(), sizeof(fl), cudaMemcpyDeviceToHost, s));
        if (tail_later) GX_CUDA(cudaMemcpyAsync(tail, uoff.get<int64_t>() + P, sizeof(tail), cudaMemcpyDeviceToHost, s));
        GX_CUDA(cudaStreamSynchronize(s));
        if (tail_later && (int)tail[1])
            fail(GX_ETIMEOUT, "partition scatter: a bulk copy into shared memory did not complete");
        if (fl[1]) { gcap *= 8; continue; }
        unsigned long long ocount_h;
        std::memcpy(&ocount_h, reinterpret_cast<const char*>(fl) + 8, 8);
        const int64_t groups = (int64_t)ocount_h;
        if (fl[4]) {
            rec_cap = std::min<int64_t>(std::max<int64_t>(n, 1), rec_cap * 4);
            continue;
        }
        emit_groupby_output(p, orec, groups, false, 0, -1, nullptr, key_in.type, out_cap, s, out);
        return;
    }
    fail(GX_EOVERFLOW, "partition group-by spill table overflow after retries");
}

// Radix-partitions a 4/8-byte key column by R bits of the partition hash
// (the id PARTITION group-by uses: fmix of the canonical key bits), moving
// every key with its row id.  keys_out / rows_out hold n entries; partition
// p is rows [part_start[p], part_start[p + 1]) of them (2^R + 1 starts).
// Row order inside a partition is unspecified.
// One stable LSD radix-sort pass through the bulk-copy scatter (digit =
// bits [shift, shift + dbits) of the key image), for 4/8-byte keys and
// optional 4/8-byte values or row ids, every loaded column starting on a
// 16-byte boundary: `offs` are the scanned digit counts [digit][tile] of
// `tile_rows`-row tiles.  Returns false, launching nothing, when the pass
// does not fit the kernel; sets *err when a bulk copy never completed.
bool radix_pass_bulk(const void* kin, const void* vin, int kw, int vw, bool iota, int64_t n, const img_params& ip,
                     int shift, int dbits, int tile_rows, const int64_t* offs, void* kout, void* vout, int* err,
                     cudaStream_t s) {
    if (getenv("GX_RADIX_NO_BULK") || tile_rows != PS_TILE || n <= 0) return false;
    if ((kw != 4 && kw != 8) || (vw != 0 && vw != 4 && vw != 8) || (iota && vw != 8)) return false;
    move_cols mc;
    std::memset(&mc, 0, sizeof(mc));
    mc.n = vw ? 2 : 1;
    mc.in[0] = kin; mc.width[0] = kw; mc.out[0] = kout;
    if (vw) { mc.in[1] = iota ? nullptr : vin; mc.width[1] = vw; mc.iota[1] = iota ? 1 : 0; mc.out[1] = vout; }
    const pb_layout L = pb_make_layout(mc, true);
    if (!bulk_scatter_ok(mc, L)) return false;
    static per_device_flag battr;
    battr.once([] {
        const int lim = dev().max_smem_optin - 2048;
        GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<4, 1, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<4, 2, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<8, 1, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        GX_CUDA(cudaFuncSetAttribute(k_part_scatter_bulk<8, 2, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    });
    const int64_t ntiles = ceil_div(n, PS_TILE);
    const int grid = (int)std::min<int64_t>(ntiles, dev().sm_count);
#define GX_RB_LAUNCH(K, NCV) \
    k_part_scatter_bulk<K, NCV, true, true><<<grid, PB_NT, L.total, s>>>(kin, n, ip.kind, ip, shift, dbits, ntiles, offs, mc, L, err)
    if (kw == 4 && mc.n == 1) GX_RB_LAUNCH(4, 1);
    else if (kw == 4) GX_RB_LAUNCH(4, 2);
    else if (mc.n == 1) GX_RB_LAUNCH(8, 1);
    else GX_RB_LAUNCH(8, 2);
#undef GX_RB_LAUNCH
    GX_LAUNCHED();
    return true;
}

void hash_partition_rows(const col& key, int R, void* keys_out, int64_t* rows_out, int64_t* part_start,
                         cudaStream_t s) {
    const int64_t n = key.n;
    const int kw = size_of(key.type);
    const int kind = vkind_of(key.type);
    require(kw == 4 || kw == 8, "hash partition: 4- or 8-byte keys");
    require(R >= 1 && R <= 16, "hash partition: 1..16 radix bits");
    const int P = 1 << R;
    if (n == 0) {
        fill_u64(part_start, 0, P + 1, s);
        return;
    }
    move_cols mc;
    std::memset(&mc, 0, sizeof(mc));
    mc.n = 2;
    mc.in[0] = key.data; mc.width[0] = kw; mc.out[0] = keys_out;
    mc.in[1] = nullptr;  mc.width[1] = 8;  mc.iota[1] = 1; mc.out[1] = rows_out;
    const int64_t ntiles = ceil_div(n, PS_TILE);
    dbuf counts((size_t)PS_BINS * ntiles * 8, s), offs((size_t)PS_BINS * ntiles * 8 + 8, s), flag(8, s);
    GX_CUDA(cudaMemsetAsync(flag.get(), 0, 8, s));
    const int passes = (R + 7) / 8;
    dbuf tk, tr;
    if (passes == 2) { tk = dbuf((size_t)n * kw, s); tr = dbuf((size_t)n * 8, s); }
    int shift = 0;
    for (int ps = 0; ps < passes; ++ps) {
        const int dbits = std::min(8, R - shift);
        move_cols m = mc;
        if (passes == 2 && ps == 0) { m.out[0] = tk.get(); m.out[1] = tr.get(); }
        if (passes == 2 && ps == 1) { m.in[0] = tk.get(); m.in[1] = tr.get(); m.iota[1] = 0; }
        if (kw == 4) part_pass<4>(m.in[0], n, kind, shift, dbits, m, counts.get<int64_t>(), offs.get<int64_t>(), flag.get<int>(), ps > 0, s);
        else part_pass<8>(m.in[0], n, kind, shift, dbits, m, counts.get<int64_t>(), offs.get<int64_t>(), flag.get<int>(), ps > 0, s);
        shift += dbits;
    }
    if (passes == 1) {
        k_starts_from_offsets<<<(unsigned)ceil_div(P + 1, 256), 256, 0, s>>>(offs.get<int64_t>(), ntiles, P, n, part_start);
        GX_LAUNCHED();
    } else {
        partition_starts(keys_out, kw, n, kind, R, part_start, s);
    }
    if (read_scalar(flag.get<int>(), s)) fail(GX_ETIMEOUT, "hash partition: a bulk copy into shared memory did not complete");
}

namespace {
template <int KW>
__global__ void k_part_starts(const void* __restrict__ keys, int64_t n, int kind, int R, int64_t* __restrict__ ps, int P) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
        int cur = i < n ? (int)(part_hash<KW>(ld_key<KW>(keys, i, kind)) & (P - 1)) : P;
        int prev = i > 0 ? (int)(part_hash<KW>(ld_key<KW>(keys, i - 1, kind)) & (P - 1)) : -1;
        for (int p = prev + 1; p <= cur; ++p) ps[p] = i;
    }
}
}  // namespace

void partition_starts(const void* keys, int kw, int64_t n, int kind, int R, int64_t* ps, cudaStream_t s) {
    int P = 1 << R;
    if (kw == 4) k_part_starts<4><<<grid_for(n + 1, 256, 8), 256, 0, s>>>(keys, n, kind, R, ps, P);
    else k_part_starts<8><<<grid_for(n + 1, 256, 8), 256, 0, s>>>(keys, n, kind, R, ps, P);
    GX_LAUNCHED();
}

}  // namespace gx
