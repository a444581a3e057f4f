// gx_groupby_sort.cu — sort-based group-by (SORT, SORT_OPT, SORT_GFUR).
//
// Replaces gamax::groupby::sort::groupby / groupby_gfur
// (src/cuda/operators/groupby/groupby_sort.cu:346-479), which sorts
// (key, value_i) once per aggregation and runs CUB ReduceByKey on each.  Here:
//   1. the key range is measured and the radix sort runs only over the bits
//      that vary (what SORT_OPT approximates with dictionary codes);
//   2. with one value column the (key, value) pairs are sorted together
//      (GFTR); otherwise (key, row id) is sorted and the values are gathered
//      through the permutation (GFUR);
//   3. one segmented-reduction kernel walks the sorted run: each thread
//      accumulates its contiguous rows in registers and flushes a group's
//      partial result with atomics only when a run ends — every group is
//      touched by at most (threads spanning it) atomics, not one per row.
// Output is ascending by key, like the reference's sort path.
#include <algorithm>

#include "gx_groupby.h"

namespace gx {

void radix_sort_biased(const col& keys_c, const void* vals_in, int val_width, bool vals_iota,
                       int begin_bit, int end_bit, bool descending, uint64_t bias, void* keys_out,
                       void* vals_out, void* temp, size_t temp_bytes, cudaStream_t s);

namespace {

constexpr int SEG_NT = 256;
constexpr int SEG_IPT = 8;
constexpr int SEG_TILE = SEG_NT * SEG_IPT;

template <int KW>
__device__ __forceinline__ uint64_t load_raw(const void* p, int64_t i) {
    if (KW == 8) return static_cast<const unsigned long long*>(p)[i];
    if (KW == 4) return static_cast<const unsigned*>(p)[i];
    if (KW == 2) return static_cast<const uint16_t*>(p)[i];
    return static_cast<const uint8_t*>(p)[i];
}
template <int KW>
__device__ __forceinline__ uint64_t canon_raw(uint64_t b, int kind) {
    if (KW == 8) return canon64(b, kind);
    if (KW == 4) return canon32((uint32_t)b, kind);
    return b;
}

template <int KW>
__global__ void __launch_bounds__(SEG_NT) k_seg_count(const void* __restrict__ skeys, int64_t n, int kind,
                                                       int64_t* __restrict__ tile_counts) {
    int64_t base = blockIdx.x * (int64_t)SEG_TILE + threadIdx.x * SEG_IPT;
    int c = 0;
    uint64_t prev = base > 0 && base <= n ? canon_raw<KW>(load_raw<KW>(skeys, base - 1), kind) : 0;
#pragma unroll
    for (int k = 0; k < SEG_IPT; ++k) {
        int64_t i = base + k;
        if (i < n) {
            uint64_t cur = canon_raw<KW>(load_raw<KW>(skeys, i), kind);
            c += (i == 0 || cur != prev);
            prev = cur;
        }
    }
    int tot = 0;
    __shared__ int sm[SEG_NT / 32];
    int w = dev_::warp_sum(c);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 0; j < SEG_NT / 32; ++j) tot += sm[j];
        tile_counts[blockIdx.x] = tot;
    }
}

// vals_mode: 0 = values sorted alongside (pairs, one column), 1 = gather through perm.
template <int KW>
__global__ void __launch_bounds__(SEG_NT) k_seg_reduce(const void* __restrict__ skeys,
                                                        const void* __restrict__ svals,
                                                        const int64_t* __restrict__ perm, int64_t n,
                                                        int kind, agg_desc d,
                                                        const int64_t* __restrict__ tile_gid,
                                                        uint64_t* __restrict__ recs) {
    __shared__ int64_t sm[SEG_NT / 32 + 1];
    int64_t base = blockIdx.x * (int64_t)SEG_TILE + threadIdx.x * SEG_IPT;
    // Run starts owned by this thread.
    int c = 0;
    uint64_t prev = base > 0 && base <= n ? canon_raw<KW>(load_raw<KW>(skeys, base - 1), kind) : 0;
    uint64_t kb[SEG_IPT];
#pragma unroll
    for (int k = 0; k < SEG_IPT; ++k) {
        int64_t i = base + k;
        kb[k] = 0;
        if (i < n) {
            kb[k] = canon_raw<KW>(load_raw<KW>(skeys, i), kind);
            c += (i == 0 || kb[k] != prev);
            prev = kb[k];
        }
    }
    int64_t total;
    int64_t gid = tile_gid[blockIdx.x] + dev_::block_exclusive_sum<SEG_NT, int64_t>(c, sm, &total) - 1;
    // gid is the group of the row before the first run start (or -1).
    uint64_t acc[MAX_ACCS];
    unsigned long long cnt = 0;
    bool open = false;
    int64_t cur_gid = gid;
    prev = base > 0 && base <= n ? canon_raw<KW>(load_raw<KW>(skeys, base - 1), kind) : 0;
    auto flush = [&]() {
        if (!open) return;
        uint64_t* r = recs + cur_gid * d.rec_words;
        if (d.has_count) atomicAdd((unsigned long long*)(r + d.count_word), cnt);
        for (int a = 0; a < d.n_acc; ++a) dev_::acc_atomic(r + d.acc_word0 + a, d.acc_op[a], d.acc_kind[a], acc[a]);
    };
    for (int k = 0; k < SEG_IPT; ++k) {
        int64_t i = base + k;
        if (i >= n) break;
        bool start = (i == 0 || kb[k] != prev);
        prev = kb[k];
        if (start || !open) {
            flush();
            if (start) {
                ++cur_gid;
                recs[cur_gid * d.rec_words] = load_raw<KW>(skeys, i);
            }
            open = true;
            cnt = 0;
            for (int a = 0; a < d.n_acc; ++a) {
                int op = d.acc_op[a], kd = d.acc_kind[a];
                acc[a] = op == OP_MIN ? (kd == VK_I ? 0x7FFFFFFFFFFFFFFFull : (kd == VK_U ? ~0ull : 0x7FF0000000000000ull))
                       : op == OP_MAX ? (kd == VK_I ? 0x8000000000000000ull : (kd == VK_U ? 0ull : 0xFFF0000000000000ull))
                       : 0ull;
            }
        }
        ++cnt;
        uint64_t v[MAX_VCOLS];
        if (perm) {
            int64_t src = perm[i];
#pragma unroll
            for (int cc = 0; cc < MAX_VCOLS; ++cc)
                if (cc < d.n_cols) v[cc] = dev_::load_lane(d.col_ptr[cc], d.col_width[cc], d.col_kind[cc], src);
        } else {
#pragma unroll
            for (int cc = 0; cc < MAX_VCOLS; ++cc)
                if (cc < d.n_cols) v[cc] = dev_::load_lane(svals, d.col_width[0], d.col_kind[0], i);
        }
        for (int a = 0; a < d.n_acc; ++a)
            acc[a] = dev_::acc_combine(d.acc_op[a], d.acc_kind[a], acc[a], dev_::pick(v, d.acc_col[a]));
    }
    // Tail runs: the lanes of a warp cover consecutive rows, so lanes whose
    // open run is the same group are adjacent.  A segmented inclusive scan
    // over the lanes folds each such stretch into its last lane, which
    // flushes once (long runs would otherwise flush once per thread).
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long g = open ? (long long)cur_gid : -2 - (long long)(blockIdx.x * (int64_t)SEG_NT + threadIdx.x);
    const long long g_next = __shfl_down_sync(FULL, g, 1);
    const bool shares_next = lane < 31 && g_next == g;
    if (__ballot_sync(FULL, shares_next) != 0) {
        for (int off = 1; off < 32; off <<= 1) {
            const long long g_up = __shfl_up_sync(FULL, g, off);
            const unsigned long long c_up = __shfl_up_sync(FULL, cnt, off);
            const bool take = lane >= off && g_up == g;
            for (int a = 0; a < d.n_acc; ++a) {
                const uint64_t a_up = __shfl_up_sync(FULL, (unsigned long long)acc[a], off);
                if (take) acc[a] = dev_::acc_combine(d.acc_op[a], d.acc_kind[a], acc[a], a_up);
            }
            if (take) cnt += c_up;
        }
        if (shares_next) return;  // a later lane holds the combined run
    }
    flush();
}

}  // namespace

void sort_groupby(const col& key, const agg_plan& p, gx_groupby_hint* hint, bool gfur, cudaStream_t s,
                  gx_table* out) {
    const int64_t n = key.n;
    const int kw = size_of(key.type);
    require(kw > 0, "SORT groupby: numeric key column required");
    int kind = vkind_of(key.type);
    // Bits that vary: sort on (image - min) over ceil(log2(max - min + 1)) bits.
    uint64_t lo = 0, hi = 0;
    int nbits = 8 * kw;
    if (n > 0 && kw >= 4) {
        key_image_range(key, &lo, &hi, s);
        uint64_t span = hi - lo;
        nbits = span == 0 ? 1 : 64 - __builtin_clzll(span);
    }
    if (kw < 4) lo = 0;
    bool pairs = !gfur && p.d.n_cols == 1 && (p.d.col_width[0] == 4 || p.d.col_width[0] == 8);
    dbuf skeys((size_t)std::max<int64_t>(n, 1) * kw, s);
    dbuf svals((size_t)std::max<int64_t>(n, 1) * 8, s);
    if (n > 0) {
        if (pairs)
            radix_sort_biased(key, p.d.col_ptr[0], p.d.col_width[0], false, 0, nbits, false, lo,
                              skeys.get(), svals.get(), nullptr, 0, s);
        else
            radix_sort_biased(key, nullptr, 8, true, 0, nbits, false, lo, skeys.get(), svals.get(), nullptr,
                              0, s);
    }
    int64_t ntiles = ceil_div(std::max<int64_t>(n, 1), SEG_TILE);
    dbuf tc(ntiles * 8, s), tg((ntiles + 1) * 8, s);
    int64_t groups = 0;
    if (n > 0) {
#define GX_SEG_COUNT(K) k_seg_count<K><<<(unsigned)ntiles, SEG_NT, 0, s>>>(skeys.get(), n, kind, tc.get<int64_t>())
        if (kw == 8) GX_SEG_COUNT(8); else if (kw == 4) GX_SEG_COUNT(4); else if (kw == 2) GX_SEG_COUNT(2); else GX_SEG_COUNT(1);
#undef GX_SEG_COUNT
        GX_LAUNCHED();
        exclusive_scan_i64(tc.get<int64_t>(), tg.get<int64_t>(), ntiles, s);
        groups = read_scalar(tg.get<int64_t>() + ntiles, s);
    }
    dbuf recs((size_t)std::max<int64_t>(groups, 1) * p.d.rec_words * 8, s);
    init_records(recs.get<uint64_t>(), groups, p.d, 0, s);
    if (n > 0) {
        const int64_t* perm = pairs ? nullptr : svals.get<int64_t>();
#define GX_SEG_RED(K) k_seg_reduce<K><<<(unsigned)ntiles, SEG_NT, 0, s>>>(skeys.get(), svals.get(), perm, n, kind, p.d, tg.get<int64_t>(), recs.get<uint64_t>())
        GX_PROF("segmented_reduce", s);
        if (kw == 8) GX_SEG_RED(8); else if (kw == 4) GX_SEG_RED(4); else if (kw == 2) GX_SEG_RED(2); else GX_SEG_RED(1);
#undef GX_SEG_RED
        GX_LAUNCHED();
    }
    int64_t out_cap = std::min<int64_t>(n, hint->groups_upper_bound > 0 ? hint->groups_upper_bound : n);
    emit_groupby_output(p, recs.get<uint64_t>(), groups, false, 0, -1, nullptr, key.type, out_cap, s, out);
}

}  // namespace gx
