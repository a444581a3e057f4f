// gx_join.cu — sort-based inner equi-join.
//
// Replaces gamax::join::inner_eq_join for join_algo SORT
// (src/cuda/operators/join/inner_join.cu:206-229, sort_merge_join.cu:111-293,
// merge_path.cuh:22-309).  The reference sorts both sides with CUB, matches
// them with a merge-path kernel that appends to a circular buffer through a
// global atomic (nondeterministic order, silent wrap past the allocation)
// and synchronises on the default stream.
//
// B200 design (GX_JOIN_SORTED_BUILD, the default):
//   1. the smaller side ("build") is radix-sorted on the bits its keys span,
//      together with its payload (one payload column) or its row id;
//   2. a radix directory over the sorted run maps the top D bits of a key's
//      image to the run's bucket, so the sorted run + directory (≈ 96 MB for
//      2^24 int32 keys) stay L2-resident;
//   3. the other side ("probe") is streamed once in its stored order: a
//      count kernel sizes every tile's output exactly, an exclusive scan
//      places the tiles, and a write kernel emits every (build, probe) pair
//      in probe order — deterministic, no wrap, no atomics.
// GX_JOIN_SORT_MERGE sorts the probe side too (key + row id) and runs the
// same matcher over the sorted stream: the reference's sort-both-sides
// structure, kept for comparison.
#include <algorithm>

#include "gx_join.h"

namespace gx {

void radix_sort_biased(const col& keys_c, const void* vals_in, int val_width, bool vals_iota,
                       int begin_bit, int end_bit, bool descending, uint64_t bias, void* keys_out,
                       void* vals_out, void* temp, size_t temp_bytes, cudaStream_t s);

namespace {

constexpr int JP_NT = 256;
constexpr int JP_IPT = 16;  // 16 rows per thread: 4096-row tiles (measured best of 8/16/32)
constexpr int JP_TILE = JP_NT * JP_IPT;

template <int KW>
__device__ __forceinline__ uint64_t img_of(const void* p, int64_t i, int kind) {
    if (KW == 4) return ordered32(__ldg(static_cast<const unsigned*>(p) + i), kind);
    return ordered64(__ldg(static_cast<const unsigned long long*>(p) + i), kind);
}

struct build_run {
    const void* keys;      // sorted build keys (raw)
    const void* vals;      // sorted build payload (or row ids)
    int val_width;         // 4 / 8
    const uint32_t* dir;   // 2^D + 1 bucket starts
    int64_t n;
    uint64_t lo, hi;       // image range of build keys
    int shift;             // bucket = (img - lo) >> shift
    int kind;
};

// Matches of IPT probe rows against the sorted build run, with the loads of
// all rows issued together (directory, then up to four keys of each small
// bucket) so their L2 latencies overlap.  Equal keys share a bucket, so a
// row's matches are the equal keys inside its bucket.
template <int KW, int IPT>
__device__ __forceinline__ void lookup_batch(const build_run& b, const uint64_t (&img)[IPT],
                                             const bool (&valid)[IPT], int64_t (&first)[IPT], int (&cnt)[IPT]) {
    uint32_t d0[IPT], d1[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        d0[k] = d1[k] = 0;
        if (valid[k] && img[k] >= b.lo && img[k] <= b.hi) {
            uint64_t bk = (img[k] - b.lo) >> b.shift;
            d0[k] = __ldg(b.dir + bk);
            d1[k] = __ldg(b.dir + bk + 1);
        }
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        first[k] = d0[k];
        cnt[k] = 0;
        uint32_t len = d1[k] - d0[k];
        if (len <= 4) {
            uint64_t kv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) kv[j] = (uint32_t)j < len ? img_of<KW>(b.keys, (int64_t)d0[k] + j, b.kind) : ~img[k];
            int f = 4, c = 0;
#pragma unroll
            for (int j = 3; j >= 0; --j)
                if (kv[j] == img[k]) { f = j; ++c; }
            first[k] = (int64_t)d0[k] + f;
            cnt[k] = c;
        } else {
            // lower and upper bound inside the bucket
            int64_t lo = d0[k], hi = d1[k];
            while (lo < hi) {
                int64_t mid = (lo + hi) >> 1;
                if (img_of<KW>(b.keys, mid, b.kind) < img[k]) lo = mid + 1;
                else hi = mid;
            }
            int64_t lo2 = lo, hi2 = d1[k];
            while (lo2 < hi2) {
                int64_t mid = (lo2 + hi2) >> 1;
                if (img_of<KW>(b.keys, mid, b.kind) <= img[k]) lo2 = mid + 1;
                else hi2 = mid;
            }
            first[k] = lo;
            cnt[k] = (int)(lo2 - lo);
        }
    }
}

struct probe_side {
    const void* keys;     // probe keys in stream order
    const int64_t* rowid; // SORT_MERGE: probe row id of stream position (else null)
    int64_t n;
    int kind;
};

// Tile layout shared by the count and write kernels: warp w of the block owns
// the contiguous rows [tile + w*32*IPT, +32*IPT); row (k, lane) = k*32 + lane.
template <int KW>
__device__ __forceinline__ void load_probe(const probe_side& p, int64_t row0, uint64_t (&img)[JP_IPT],
                                           bool (&valid)[JP_IPT]) {
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) {
        int64_t i = row0 + k * 32;
        valid[k] = i < p.n;
        img[k] = valid[k] ? img_of<KW>(p.keys, i, p.kind) : 0;
    }
}

template <int KW>
__global__ void __launch_bounds__(JP_NT) k_probe_count(build_run b, probe_side p, int64_t* __restrict__ tile_out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int64_t row0 = blockIdx.x * (int64_t)JP_TILE + warp * 32 * JP_IPT + lane;
    uint64_t img[JP_IPT];
    bool valid[JP_IPT];
    int64_t first[JP_IPT];
    int cnt[JP_IPT];
    load_probe<KW>(p, row0, img, valid);
    lookup_batch<KW, JP_IPT>(b, img, valid, first, cnt);
    int64_t c = 0;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) c += cnt[k];
    __shared__ int64_t sm[JP_NT / 32];
    c = dev_::warp_sum(c);
    if (lane == 0) sm[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int j = 0; j < JP_NT / 32; ++j) t += sm[j];
        tile_out[blockIdx.x] = t;
    }
}

template <int KW>
__global__ void __launch_bounds__(JP_NT) k_probe_write(build_run b, probe_side p, const int64_t* __restrict__ tile_off,
                                                        join_out o) {
    __shared__ int64_t sm[JP_NT / 32 + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int64_t row0 = blockIdx.x * (int64_t)JP_TILE + warp * 32 * JP_IPT + lane;
    uint64_t img[JP_IPT];
    bool valid[JP_IPT];
    int64_t first[JP_IPT];
    int cnt[JP_IPT];
    load_probe<KW>(p, row0, img, valid);
    lookup_batch<KW, JP_IPT>(b, img, valid, first, cnt);
    int64_t mine = 0;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) mine += cnt[k];
    int64_t wtot = dev_::warp_sum(mine);
    // Exclusive prefix over the warps of the tile (warp-major = row order).
    int64_t total;
    int64_t wbase = dev_::block_exclusive_sum<JP_NT, int64_t>(lane == 0 ? wtot : 0, sm, &total);
    wbase = __shfl_sync(0xffffffffu, wbase, 0) + tile_off[blockIdx.x];
    int64_t running = 0;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) {
        int64_t inc = dev_::warp_inclusive_sum((int64_t)cnt[k]);
        int64_t pos = wbase + running + inc - cnt[k];
        running += __shfl_sync(0xffffffffu, inc, 31);
        int64_t i = row0 + k * 32;
        for (int m = 0; m < cnt[k]; ++m, ++pos) {
            int64_t bm = first[k] + m;
            int64_t prow = p.rowid ? p.rowid[i] : i;
            if (o.key) st_w(o.key, o.key_width, pos, ld_w(b.keys, o.key_width, bm));
            for (int c = 0; c < o.n_pay; ++c) {
                uint64_t v;
                switch (o.src[c]) {
                    case 0: v = ld_w(b.vals, b.val_width, bm); break;
                    case 1: v = ld_w(o.col[c], o.width[c], (int64_t)ld_w(b.vals, 8, bm)); break;
                    case 2: v = ld_w(o.col[c], o.width[c], prow); break;
                    case 3: v = ld_w(b.vals, 8, bm); break;
                    default: v = (uint64_t)prow; break;
                }
                st_w(o.out[c], o.width[c], pos, v);
            }
        }
    }
}

template <int KW>
__global__ void k_build_dir(const void* __restrict__ skeys, int64_t n, int kind, uint64_t lo, int shift,
                            uint64_t nb, uint32_t* __restrict__ dir, int* __restrict__ dup) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t ci = i < n ? img_of<KW>(skeys, i, kind) : 0, pi = i > 0 ? img_of<KW>(skeys, i - 1, kind) : 0;
        uint64_t cur = i < n ? (ci - lo) >> shift : nb;
        uint64_t prev = i > 0 ? (pi - lo) >> shift : (uint64_t)-1;
        for (uint64_t j = prev + 1; j <= cur; ++j) dir[j] = (uint32_t)i;
        if (i > 0 && i < n && ci == pi) *dup = 1;  // equal neighbours: build keys are not unique
    }
}

struct sorted_side {
    dbuf keys, vals;
    int val_width = 8;
    bool vals_are_payload = false;
};

}  // namespace

// ---------------------------------------------------------------------------
// Dense unique build keys.  When the build keys are unique and span at most
// four times their count, ordering them is a counting sort whose rank is the
// key itself: row i lands at position image(key_i) - min.  The placed row ids
// (uint32, 4 B per position: 64 MB for 2^24 keys) stay L2-resident, and a
// probe row finds its match with one L2 read instead of a search.
// ---------------------------------------------------------------------------
constexpr uint32_t NO_ROW = 0xFFFFFFFFu;

template <int KW>
__global__ void k_dense_place(const void* __restrict__ keys, int64_t n, int kind, uint64_t lo,
                              uint32_t* __restrict__ slot_row, int* __restrict__ dup) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t pos = img_of<KW>(keys, i, kind) - lo;
        uint32_t old = atomicCAS(slot_row + pos, NO_ROW, (uint32_t)i);
        if (old != NO_ROW) atomicExch(dup, 1);
    }
}

template <int KW>
__device__ __forceinline__ void dense_lookup(const void* pkeys, int64_t np, int kind, uint64_t lo, uint64_t hi,
                                             const uint32_t* slot_row, int64_t row0, uint32_t (&m)[JP_IPT]) {
    // Probe keys are read once: load them with the streaming (evict-first)
    // hint so they do not push the placement array out of L2.
    uint64_t img[JP_IPT];
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) {
        int64_t i = row0 + k * 32;
        if (i < np) {
            if (KW == 4) img[k] = ordered32(__ldcs(static_cast<const unsigned*>(pkeys) + i), kind);
            else img[k] = ordered64(__ldcs(static_cast<const unsigned long long*>(pkeys) + i), kind);
        } else {
            img[k] = hi + 1;
        }
    }
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k)
        m[k] = (img[k] >= lo && img[k] <= hi) ? __ldg(slot_row + (img[k] - lo)) : NO_ROW;
}

template <int KW>
__global__ void __launch_bounds__(JP_NT) k_dense_count(const void* __restrict__ pkeys, int64_t np, int kind,
                                                        uint64_t lo, uint64_t hi,
                                                        const uint32_t* __restrict__ slot_row,
                                                        int64_t* __restrict__ tile_out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int64_t row0 = blockIdx.x * (int64_t)JP_TILE + warp * 32 * JP_IPT + lane;
    uint32_t m[JP_IPT];
    dense_lookup<KW>(pkeys, np, kind, lo, hi, slot_row, row0, m);
    int c = 0;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) c += m[k] != NO_ROW;
    __shared__ int sm[JP_NT / 32];
    c = dev_::warp_sum(c);
    if (lane == 0) sm[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int j = 0; j < JP_NT / 32; ++j) t += sm[j];
        tile_out[blockIdx.x] = t;
    }
}

// Output sources for the dense path: 1 = build column at the build row,
// 2 = probe column at the probe row, 3 = build row id, 4 = probe row id.
template <int KW>
__global__ void __launch_bounds__(JP_NT) k_dense_write(const void* __restrict__ pkeys, int64_t np, int kind,
                                                        uint64_t lo, uint64_t hi,
                                                        const uint32_t* __restrict__ slot_row,
                                                        const int64_t* __restrict__ tile_off, join_out o) {
    __shared__ int64_t sm[JP_NT / 32 + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int64_t row0 = blockIdx.x * (int64_t)JP_TILE + warp * 32 * JP_IPT + lane;
    uint32_t m[JP_IPT];
    dense_lookup<KW>(pkeys, np, kind, lo, hi, slot_row, row0, m);
    int c = 0;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) c += m[k] != NO_ROW;
    int64_t wtot = dev_::warp_sum((int64_t)c);
    int64_t total;
    int64_t wbase = dev_::block_exclusive_sum<JP_NT, int64_t>(lane == 0 ? wtot : 0, sm, &total);
    wbase = __shfl_sync(0xffffffffu, wbase, 0) + tile_off[blockIdx.x];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) {
        bool hit = m[k] != NO_ROW;
        unsigned bal = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            int64_t pos = wbase + __popc(bal & lt);
            int64_t i = row0 + k * 32;
            if (o.key) st_w(o.key, o.key_width, pos, ld_w(pkeys, o.key_width, i));
            for (int cc = 0; cc < o.n_pay; ++cc) {
                uint64_t v;
                switch (o.src[cc]) {
                    case 1: v = ld_w(o.col[cc], o.width[cc], (int64_t)m[k]); break;
                    case 2: v = ld_w(o.col[cc], o.width[cc], i); break;
                    case 3: v = (uint64_t)m[k]; break;
                    default: v = (uint64_t)i; break;
                }
                st_w(o.out[cc], o.width[cc], pos, v);
            }
        }
        wbase += __popc(bal);
    }
}

// ---------------------------------------------------------------------------
// Single-pass dense probe: count, place and write in one kernel.  With unique
// build keys a probe row has at most one match, so the output fits in
// `np` rows and can be allocated before the probe.  Tiles take their index
// from an atomic ticket (so every tile a block waits on belongs to a block
// that started earlier), publish their match count, and find their output
// start by a decoupled look-back over the predecessors' published counts
// (Merrill & Garland, "Single-pass Parallel Prefix Scan with Decoupled
// Look-back", NVIDIA TR 2016).  Probe keys are read and looked up once
// instead of twice.  Every wait is bounded: a tile that gives up sets *err,
// publishes anyway so its successors do not wait on it, and writes nothing;
// the host then reruns the two-pass probe.
// ---------------------------------------------------------------------------
constexpr unsigned long long TS_AGG = 1ull << 62, TS_INC = 2ull << 62, TS_VAL = (1ull << 62) - 1;
constexpr int LOOKBACK_SPIN_LIMIT = 1 << 20;

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Exclusive output start of `tile` (warp 0 calls it; all lanes get the value).
__device__ __forceinline__ int64_t lookback(unsigned long long* tstate, int64_t tile, int64_t total, int* err) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) st_release_u64(tstate, TS_INC | (unsigned long long)total);
        return 0;
    }
    if (lane == 0) st_release_u64(tstate + tile, TS_AGG | (unsigned long long)total);
    int64_t excl = 0, end = tile - 1;  // lane j looks at tile end - j
    int spins = 0;
    while (true) {
        int64_t j = end - lane;
        unsigned long long st = j >= 0 ? ld_acquire_u64(tstate + j) : TS_INC;
        unsigned inc = __ballot_sync(0xffffffffu, (st >> 62) == 2);
        unsigned none = __ballot_sync(0xffffffffu, (st >> 62) == 0);
        int stop = inc ? __ffs(inc) - 1 : 31;  // nearest inclusive predecessor, else the whole window
        unsigned need = stop == 31 ? 0xffffffffu : ((2u << stop) - 1u);
        if (none & need) {
            if (++spins > LOOKBACK_SPIN_LIMIT) {
                if (lane == 0) atomicExch(err, 1);
                break;
            }
            __nanosleep(32);
            continue;
        }
        int64_t v = (lane <= stop && j >= 0) ? (int64_t)(st & TS_VAL) : 0;
        excl += dev_::warp_sum(v);
        if (inc) break;
        end -= 32;
    }
    if (lane == 0) st_release_u64(tstate + tile, TS_INC | (unsigned long long)(excl + total));
    return excl;
}

// ROWIDS: the output is just the (build row, probe row) pair (int64 each).
template <int KW, bool ROWIDS>
__global__ void __launch_bounds__(JP_NT) k_dense_probe1(const void* __restrict__ pkeys, int64_t np, int kind,
                                                         uint64_t lo, uint64_t hi,
                                                         const uint32_t* __restrict__ slot_row,
                                                         unsigned long long* __restrict__ tstate,
                                                         unsigned* __restrict__ ticket, int64_t ntiles,
                                                         int64_t* __restrict__ total_out, int* __restrict__ err,
                                                         join_out o) {
    __shared__ int64_t sm[JP_NT / 32 + 1];
    __shared__ int64_t s_tile, s_excl;
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const int64_t tile = s_tile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int64_t row0 = tile * (int64_t)JP_TILE + warp * 32 * JP_IPT + lane;
    uint32_t m[JP_IPT];
    dense_lookup<KW>(pkeys, np, kind, lo, hi, slot_row, row0, m);
    int c = 0;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) c += m[k] != NO_ROW;
    int64_t wtot = dev_::warp_sum((int64_t)c);
    int64_t total;
    int64_t wbase = dev_::block_exclusive_sum<JP_NT, int64_t>(lane == 0 ? wtot : 0, sm, &total);
    if (warp == 0) {
        int64_t excl = lookback(tstate, tile, total, err);
        __syncwarp();  // orders the lanes' acquire loads before lane 0 reads the error flag
        if (lane == 0) {
            s_excl = excl;
            s_skip = *(volatile int*)err;
            if (tile == ntiles - 1) *total_out = excl + total;
        }
    }
    __syncthreads();
    if (s_skip) return;  // block-uniform
    wbase = __shfl_sync(0xffffffffu, wbase, 0) + s_excl;
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) {
        bool hit = m[k] != NO_ROW;
        unsigned bal = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            int64_t pos = wbase + __popc(bal & lt);
            int64_t i = row0 + k * 32;
            if (pos < np) {  // capacity bound (a unique-key probe never exceeds it)
                if constexpr (ROWIDS) {
                    // Output rows are written once: streaming stores keep them
                    // from evicting the placement array.
                    const int64_t b = (int64_t)m[k];
                    const bool build_first = o.src[0] == 3;
                    __stcs(static_cast<long long*>(o.out[0]) + pos, (long long)(build_first ? b : i));
                    __stcs(static_cast<long long*>(o.out[1]) + pos, (long long)(build_first ? i : b));
                } else {
                    if (o.key) st_w(o.key, o.key_width, pos, ld_w(pkeys, o.key_width, i));
                    for (int cc = 0; cc < o.n_pay; ++cc) {
                        uint64_t v;
                        switch (o.src[cc]) {
                            case 1: v = ld_w(o.col[cc], o.width[cc], (int64_t)m[k]); break;
                            case 2: v = ld_w(o.col[cc], o.width[cc], i); break;
                            case 3: v = (uint64_t)m[k]; break;
                            default: v = (uint64_t)i; break;
                        }
                        st_w(o.out[cc], o.width[cc], pos, v);
                    }
                }
            }
        }
        wbase += __popc(bal);
    }
}

// Single-pass probe of the sorted build run for unique build keys (at most
// one match per probe row, so the outputs are allocated for every probe row
// up front): the tile's matches are placed with the decoupled look-back of
// k_dense_probe1 instead of a count kernel, a scan and a second lookup.
template <int KW>
__global__ void __launch_bounds__(JP_NT) k_sorted_probe1(build_run b, probe_side p, unsigned long long* __restrict__ tstate,
                                                        unsigned* __restrict__ ticket, int64_t ntiles,
                                                        int64_t* __restrict__ total_out, int* __restrict__ err,
                                                        join_out o) {
    __shared__ int64_t sm[JP_NT / 32 + 1];
    __shared__ int64_t s_tile, s_excl;
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const int64_t tile = s_tile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row0 = tile * (int64_t)JP_TILE + warp * 32 * JP_IPT + lane;
    uint64_t img[JP_IPT];
    bool valid[JP_IPT];
    int64_t first[JP_IPT];
    int cnt[JP_IPT];
    load_probe<KW>(p, row0, img, valid);
    lookup_batch<KW, JP_IPT>(b, img, valid, first, cnt);
    int c = 0;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) c += cnt[k] > 0;
    const int64_t wtot = dev_::warp_sum((int64_t)c);
    int64_t total;
    int64_t wbase = dev_::block_exclusive_sum<JP_NT, int64_t>(lane == 0 ? wtot : 0, sm, &total);
    if (warp == 0) {
        const int64_t excl = lookback(tstate, tile, total, err);
        __syncwarp();  // orders the lanes' acquire loads before lane 0 reads the error flag
        if (lane == 0) {
            s_excl = excl;
            s_skip = *(volatile int*)err;
            if (tile == ntiles - 1) *total_out = excl + total;
        }
    }
    __syncthreads();
    if (s_skip) return;  // block-uniform
    wbase = __shfl_sync(0xffffffffu, wbase, 0) + s_excl;
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < JP_IPT; ++k) {
        const bool hit = cnt[k] > 0;
        const unsigned bal = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const int64_t pos = wbase + __popc(bal & lt);
            const int64_t i = row0 + k * 32;
            if (pos < p.n) {  // capacity bound (unique build keys never exceed it)
                const int64_t bm = first[k];
                const int64_t prow = p.rowid ? p.rowid[i] : i;
                if (o.key) st_w(o.key, o.key_width, pos, ld_w(b.keys, o.key_width, bm));
                for (int cc = 0; cc < o.n_pay; ++cc) {
                    uint64_t v;
                    switch (o.src[cc]) {
                        case 0: v = ld_w(b.vals, b.val_width, bm); break;
                        case 1: v = ld_w(o.col[cc], o.width[cc], (int64_t)ld_w(b.vals, 8, bm)); break;
                        case 2: v = ld_w(o.col[cc], o.width[cc], prow); break;
                        case 3: v = ld_w(b.vals, 8, bm); break;
                        default: v = (uint64_t)prow; break;
                    }
                    st_w(o.out[cc], o.width[cc], pos, v);
                }
            }
        }
        wbase += __popc(bal);
    }
}

// Output columns of a join: [key, left payloads.., right payloads..] or the
// row-id pair; `dense` selects the source codes of the dense path.
join_out make_outputs(const join_inputs& in, bool build_left, bool rowids_only, bool pay_in_run, bool dense,
                      int64_t total, cudaStream_t s, gx_table* out, int64_t cap) {
    join_out o;
    std::memset(&o, 0, sizeof(o));
    out->cols.clear();
    const int kw = size_of(in.lkey.type);
    if (rowids_only) {
        out->cols.push_back(make_col(GX_INT64, total, s, cap));
        out->cols.push_back(make_col(GX_INT64, total, s, cap));
        o.n_pay = 2;
        o.out[0] = out->cols[0].buf.get(); o.width[0] = 8; o.src[0] = build_left ? 3 : 4;
        o.out[1] = out->cols[1].buf.get(); o.width[1] = 8; o.src[1] = build_left ? 4 : 3;
        return o;
    }
    out->cols.push_back(make_col(in.lkey.type, total, s, cap));
    o.key = out->cols[0].buf.get();
    o.key_width = kw;
    auto add_side = [&](bool is_build, const std::vector<col>& pays) {
        for (size_t c = 0; c < pays.size(); ++c) {
            int w = size_of(pays[c].type);
            require(w > 0, "join: STRING payload columns are not supported");
            out->cols.push_back(make_col(pays[c].type, total, s, cap));
            int j = o.n_pay++;
            o.out[j] = out->cols.back().buf.get();
            o.width[j] = w;
            o.col[j] = pays[c].data;
            o.src[j] = is_build ? (dense ? 1 : (pay_in_run ? 0 : 1)) : 2;
        }
    };
    if (build_left) { add_side(true, in.lpay); add_side(false, in.rpay); }
    else { add_side(false, in.lpay); add_side(true, in.rpay); }
    return o;
}

// Returns false when the build keys turn out not to be unique.
static bool dense_join(const join_inputs& in, const gx_join_hint& hint, bool rowids_only, bool build_left,
                       uint64_t lo, uint64_t hi, cudaStream_t s, gx_table* out) {
    const col& bkey = build_left ? in.lkey : in.rkey;
    const col& pkey = build_left ? in.rkey : in.lkey;
    const int kw = size_of(in.lkey.type);
    const int kind = vkind_of(in.lkey.type);
    const int64_t nb = bkey.n, np = pkey.n;
    uint64_t npos = hi - lo + 1;
    dbuf slot_row((size_t)npos * 4, s), flag(8, s);
    fill_u32(slot_row.get(), NO_ROW, (int64_t)npos, s);
    GX_CUDA(cudaMemsetAsync(flag.get(), 0, 8, s));
    {
        GX_PROF("join_build_place", s);
        if (kw == 4) k_dense_place<4><<<grid_for(nb, 256, 8), 256, 0, s>>>(bkey.data, nb, kind, lo, slot_row.get<uint32_t>(), flag.get<int>());
        else k_dense_place<8><<<grid_for(nb, 256, 8), 256, 0, s>>>(bkey.data, nb, kind, lo, slot_row.get<uint32_t>(), flag.get<int>());
        GX_LAUNCHED();
    }
    if (read_scalar(flag.get<int>(), s)) return false;
    int64_t ntiles = ceil_div(std::max<int64_t>(np, 1), JP_TILE);
    static const bool two_pass = getenv("GX_JOIN_TWO_PASS") != nullptr;
    if (np > 0 && !two_pass) {
        // Unique build keys: at most np matches, so the outputs are allocated
        // up front and the probe runs once.
        dbuf tstate((size_t)ntiles * 8 + 16, s), scal(16, s);
        GX_CUDA(cudaMemsetAsync(tstate.get(), 0, (size_t)ntiles * 8 + 16, s));
        GX_CUDA(cudaMemsetAsync(scal.get(), 0, 16, s));
        join_out o = make_outputs(in, build_left, rowids_only, false, true, np, s, out, np);
        unsigned* ticket = reinterpret_cast<unsigned*>(tstate.get<char>() + (size_t)ntiles * 8);
        int64_t* total_out = scal.get<int64_t>();
        int* err = reinterpret_cast<int*>(scal.get<char>() + 8);
        {
            GX_PROF("join_probe_write", s);
#define GX_PROBE1(KW_, RID_)                                                                            \
    k_dense_probe1<KW_, RID_><<<(unsigned)ntiles, JP_NT, 0, s>>>(pkey.data, np, kind, lo, hi,              \
                                                                 slot_row.get<uint32_t>(),                \
                                                                 tstate.get<unsigned long long>(), ticket, \
                                                                 ntiles, total_out, err, o)
            if (kw == 4 && rowids_only) GX_PROBE1(4, true);
            else if (kw == 4) GX_PROBE1(4, false);
            else if (rowids_only) GX_PROBE1(8, true);
            else GX_PROBE1(8, false);
#undef GX_PROBE1
            GX_LAUNCHED();
        }
        int64_t hs[2];
        GX_CUDA(cudaMemcpyAsync(hs, scal.get(), 16, cudaMemcpyDeviceToHost, s));
        GX_CUDA(cudaStreamSynchronize(s));
        if ((int)hs[1] == 0) {
            const int64_t total = hs[0];
            if (hint.max_out > 0 && total > hint.max_out)
                fail(GX_EOVERFLOW, "join output (" + std::to_string(total) + " rows) exceeds hint.max_out (" +
                                       std::to_string(hint.max_out) + ")");
            for (auto& c : out->cols) c.size = total;
            return true;
        }
        out->cols.clear();  // a look-back wait gave up: redo with the two-pass probe
    }
    dbuf tc(ntiles * 8, s), toff((ntiles + 1) * 8, s);
    int64_t total = 0;
    if (np > 0) {
        GX_PROF("join_probe_count", s);
        if (kw == 4) k_dense_count<4><<<(unsigned)ntiles, JP_NT, 0, s>>>(pkey.data, np, kind, lo, hi, slot_row.get<uint32_t>(), tc.get<int64_t>());
        else k_dense_count<8><<<(unsigned)ntiles, JP_NT, 0, s>>>(pkey.data, np, kind, lo, hi, slot_row.get<uint32_t>(), tc.get<int64_t>());
        GX_LAUNCHED();
        exclusive_scan_i64(tc.get<int64_t>(), toff.get<int64_t>(), ntiles, s);
        total = read_scalar(toff.get<int64_t>() + ntiles, s);
    }
    if (hint.max_out > 0 && total > hint.max_out)
        fail(GX_EOVERFLOW, "join output (" + std::to_string(total) + " rows) exceeds hint.max_out (" +
                               std::to_string(hint.max_out) + ")");
    join_out o = make_outputs(in, build_left, rowids_only, false, true, total, s, out);
    if (total > 0) {
        GX_PROF("join_probe_write", s);
        if (kw == 4) k_dense_write<4><<<(unsigned)ntiles, JP_NT, 0, s>>>(pkey.data, np, kind, lo, hi, slot_row.get<uint32_t>(), toff.get<int64_t>(), o);
        else k_dense_write<8><<<(unsigned)ntiles, JP_NT, 0, s>>>(pkey.data, np, kind, lo, hi, slot_row.get<uint32_t>(), toff.get<int64_t>(), o);
        GX_LAUNCHED();
    }
    GX_CUDA(cudaStreamSynchronize(s));
    return true;
}

// Core: returns owned output columns in order [key?, left payloads.., right payloads..]
// or [left_rowid, right_rowid] when rowids_only.
static void join_core(const join_inputs& in, const gx_join_hint& hint, bool rowids_only, cudaStream_t s,
                      gx_table* out) {
    const int kw = size_of(in.lkey.type);
    require(in.lkey.type == in.rkey.type, "Join columns cannot have different types");
    require(kw == 4 || kw == 8, "join: 4- or 8-byte key columns supported");
    const int kind = vkind_of(in.lkey.type);
    // Build = smaller side.
    bool build_left = in.lkey.n <= in.rkey.n;
    const col& bkey = build_left ? in.lkey : in.rkey;
    const col& pkey = build_left ? in.rkey : in.lkey;
    const std::vector<col>& bpay = build_left ? in.lpay : in.rpay;
    const std::vector<col>& ppay = build_left ? in.rpay : in.lpay;
    require((int)bpay.size() <= MAX_PAY && (int)ppay.size() <= MAX_PAY, "join: too many payload columns");

    const int64_t nb = bkey.n, np = pkey.n;
    uint64_t lo = 0, hi = 0;
    if (nb > 0) key_image_range(bkey, &lo, &hi, s);
    uint64_t span = hi - lo;
    // Dense unique build keys: place rows by key instead of comparison sorting.
    if (nb > 0 && hint.sort_mode == GX_JOIN_SORTED_BUILD && nb < (int64_t)NO_ROW && span < (uint64_t)nb * 4 &&
        dense_join(in, hint, rowids_only, build_left, lo, hi, s, out))
        return;
    // Sort the build side: (key, payload) when exactly one 4/8-byte payload.
    bool pay_in_run = !rowids_only && bpay.size() == 1 && (size_of(bpay[0].type) == 4 || size_of(bpay[0].type) == 8);
    int vw = pay_in_run ? size_of(bpay[0].type) : 8;
    dbuf bk((size_t)std::max<int64_t>(nb, 1) * kw, s), bv((size_t)std::max<int64_t>(nb, 1) * vw, s);
    int nbits = span == 0 ? 1 : 64 - __builtin_clzll(span);
    if (nb > 0) {
        if (pay_in_run) radix_sort_biased(bkey, bpay[0].data, vw, false, 0, nbits, false, lo, bk.get(), bv.get(), nullptr, 0, s);
        else radix_sort_biased(bkey, nullptr, 8, true, 0, nbits, false, lo, bk.get(), bv.get(), nullptr, 0, s);
    }
    // Directory: D bits, about two build keys per bucket.
    int D = std::min(nbits, std::max(1, ilog2_ceil((uint64_t)std::max<int64_t>(nb, 2)) - 1));
    int shift = nbits - D;
    uint64_t nbk = (span >> shift) + 1;
    dbuf dir((size_t)(nbk + 1) * 4, s), dup(8, s);
    GX_CUDA(cudaMemsetAsync(dup.get(), 0, 8, s));
    if (nb > 0) {
        if (kw == 4) k_build_dir<4><<<grid_for(nb + 1, 256, 8), 256, 0, s>>>(bk.get(), nb, kind, lo, shift, nbk, dir.get<uint32_t>(), dup.get<int>());
        else k_build_dir<8><<<grid_for(nb + 1, 256, 8), 256, 0, s>>>(bk.get(), nb, kind, lo, shift, nbk, dir.get<uint32_t>(), dup.get<int>());
        GX_LAUNCHED();
    }
    build_run br{bk.get(), bv.get(), vw, dir.get<uint32_t>(), nb, lo, hi, shift, kind};

    // Probe stream (sorted for SORT_MERGE).
    probe_side ps{pkey.data, nullptr, np, kind};
    dbuf psk, psr;
    if (hint.sort_mode == GX_JOIN_SORT_MERGE && np > 0) {
        uint64_t plo, phi;
        key_image_range(pkey, &plo, &phi, s);
        uint64_t pspan = phi - plo;
        int pbits = pspan == 0 ? 1 : 64 - __builtin_clzll(pspan);
        psk = dbuf((size_t)np * kw, s);
        psr = dbuf((size_t)np * 8, s);
        radix_sort_biased(pkey, nullptr, 8, true, 0, pbits, false, plo, psk.get(), psr.get(), nullptr, 0, s);
        ps.keys = psk.get();
        ps.rowid = psr.get<int64_t>();
    }

    int64_t ntiles = ceil_div(std::max<int64_t>(np, 1), JP_TILE);
    static const bool two_pass = getenv("GX_JOIN_TWO_PASS") != nullptr;
    if (np > 0 && nb > 0 && !two_pass && !read_scalar(dup.get<int>(), s)) {
        // Unique build keys: one probe pass, tiles placed by look-back.
        dbuf tstate((size_t)ntiles * 8 + 16, s), scal(16, s);
        GX_CUDA(cudaMemsetAsync(tstate.get(), 0, (size_t)ntiles * 8 + 16, s));
        GX_CUDA(cudaMemsetAsync(scal.get(), 0, 16, s));
        join_out o = make_outputs(in, build_left, rowids_only, pay_in_run, false, np, s, out, np);
        unsigned* ticket = reinterpret_cast<unsigned*>(tstate.get<char>() + (size_t)ntiles * 8);
        {
            GX_PROF("join_probe_write", s);
            if (kw == 4)
                k_sorted_probe1<4><<<(unsigned)ntiles, JP_NT, 0, s>>>(br, ps, tstate.get<unsigned long long>(), ticket,
                                                                     ntiles, scal.get<int64_t>(),
                                                                     reinterpret_cast<int*>(scal.get<char>() + 8), o);
            else
                k_sorted_probe1<8><<<(unsigned)ntiles, JP_NT, 0, s>>>(br, ps, tstate.get<unsigned long long>(), ticket,
                                                                     ntiles, scal.get<int64_t>(),
                                                                     reinterpret_cast<int*>(scal.get<char>() + 8), o);
            GX_LAUNCHED();
        }
        int64_t hs[2];
        GX_CUDA(cudaMemcpyAsync(hs, scal.get(), 16, cudaMemcpyDeviceToHost, s));
        GX_CUDA(cudaStreamSynchronize(s));
        if ((int)hs[1] == 0) {
            const int64_t total = hs[0];
            if (hint.max_out > 0 && total > hint.max_out)
                fail(GX_EOVERFLOW, "join output (" + std::to_string(total) + " rows) exceeds hint.max_out (" +
                                       std::to_string(hint.max_out) + ")");
            for (auto& c : out->cols) c.size = total;
            return;
        }
        out->cols.clear();  // a look-back wait gave up: redo with the two-pass probe
    }
    dbuf tc(ntiles * 8, s), toff((ntiles + 1) * 8, s);
    int64_t total = 0;
    if (np > 0 && nb > 0) {
        GX_PROF("join_probe_count", s);
        if (kw == 4) k_probe_count<4><<<(unsigned)ntiles, JP_NT, 0, s>>>(br, ps, tc.get<int64_t>());
        else k_probe_count<8><<<(unsigned)ntiles, JP_NT, 0, s>>>(br, ps, tc.get<int64_t>());
        GX_LAUNCHED();
        exclusive_scan_i64(tc.get<int64_t>(), toff.get<int64_t>(), ntiles, s);
        total = read_scalar(toff.get<int64_t>() + ntiles, s);
    }
    if (hint.max_out > 0 && total > hint.max_out)
        fail(GX_EOVERFLOW, "join output (" + std::to_string(total) + " rows) exceeds hint.max_out (" +
                               std::to_string(hint.max_out) + ")");

    join_out o = make_outputs(in, build_left, rowids_only, pay_in_run, false, total, s, out);
    if (total > 0) {
        GX_PROF("join_probe_write", s);
        if (kw == 4) k_probe_write<4><<<(unsigned)ntiles, JP_NT, 0, s>>>(br, ps, toff.get<int64_t>(), o);
        else k_probe_write<8><<<(unsigned)ntiles, JP_NT, 0, s>>>(br, ps, toff.get<int64_t>(), o);
        GX_LAUNCHED();
    }
    GX_CUDA(cudaStreamSynchronize(s));
}

// join_algo picks the plan: SORT (dense placement or sorted build + radix
// directory, above), HASH (global multiset) or PARTITION (radix-partitioned
// shared-memory tables), the last two in gx_join_hash.cu.  All three return
// the same pair multiset.
static void run_join(const join_inputs& in, const gx_join_hint& hint, bool rowids_only, cudaStream_t s,
                     gx_table* out) {
    if (hint.join_algo == GX_JOIN_HASH) hash_join(in, hint, rowids_only, s, out);
    else if (hint.join_algo == GX_JOIN_PARTITION) partition_hash_join(in, hint, rowids_only, s, out);
    else join_core(in, hint, rowids_only, s, out);
}

void inner_eq_join(const gx_table_view* left, const gx_table_view* right, const gx_join_hint* hint,
                   cudaStream_t s, gx_table* out) {
    require(left && right && hint, "join: null argument");
    // Validation mirrors check_join_solvable (inner_join.cu:17-45).
    if (hint->join_algo == GX_JOIN_AUTO || hint->mat_algo == GX_MAT_AUTO)
        fail(GX_EINVAL, "Join algorithm and materialization algorithm do not support auto selection");
    if (hint->max_out > GX_MAX_JOIN_OUTPUT_SIZE) fail(GX_EINVAL, "Output size exceeds the maximum limit");
    if (hint->mat_algo == GX_MAT_INDEX_CLUSTER)
        fail(GX_EINVAL, "Index cluster materialization algorithm is not supported");
    if (left->num_columns == 0 || right->num_columns == 0) fail(GX_EINVAL, "Empty table");
    if (left->columns[0].type != right->columns[0].type) fail(GX_EINVAL, "Join columns cannot have different types");
    if (left->num_columns == 1 || right->num_columns == 1)
        fail(GX_EINVAL, "Left and right table should have at least 1 payload column");
    if (hint->join_algo != GX_JOIN_SORT && hint->join_algo != GX_JOIN_HASH && hint->join_algo != GX_JOIN_PARTITION)
        fail(GX_EINVAL, "Unsupported join algorithm");
    join_inputs in;
    in.lkey = resolve(left->columns[0]);
    in.rkey = resolve(right->columns[0]);
    for (int64_t c = 1; c < left->num_columns; ++c) {
        in.lpay.push_back(resolve(left->columns[c]));
        require(in.lpay.back().n == in.lkey.n, "join: left payload length differs from key length");
    }
    for (int64_t c = 1; c < right->num_columns; ++c) {
        in.rpay.push_back(resolve(right->columns[c]));
        require(in.rpay.back().n == in.rkey.n, "join: right payload length differs from key length");
    }
    run_join(in, *hint, false, s, out);
}

void inner_eq_join_rowids(const gx_column_view& l, const gx_column_view& r, const gx_join_hint* hint,
                          cudaStream_t s, gx_table* out) {
    join_inputs in;
    in.lkey = resolve(l);
    in.rkey = resolve(r);
    gx_join_hint h;
    if (hint) h = *hint;
    else { std::memset(&h, 0, sizeof(h)); h.join_algo = GX_JOIN_SORT; h.mat_algo = GX_MAT_GFUR; }
    if (h.max_out > GX_MAX_JOIN_OUTPUT_SIZE) fail(GX_EINVAL, "Output size exceeds the maximum limit");
    run_join(in, h, true, s, out);
}

}  // namespace gx
