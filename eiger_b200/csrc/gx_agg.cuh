// gx_agg.cuh — aggregation plan shared by the hash, sort and partition
// group-by variants: request rewriting, accumulator encoding, device-side
// update/merge primitives and the record -> output column conversion.
//
// Semantics follow the reference:
//   * request rewriting AVG -> SUM + COUNT, COUNT_ALL / agg_count -> COUNT
//     (src/cuda/operators/groupby/groupby.cu:128-244);
//   * output types: SUM(int8..int64) -> INT64, SUM(uint8..uint32) -> UINT64,
//     SUM(float) -> FLOAT32, SUM(double) -> FLOAT64, MIN/MAX/ANY keep the input
//     type, AVG -> FLOAT64, COUNT -> INT64
//     (src/cuda/operators/groupby/agg_func.cuh:20-35, aggregate.cu:19-53);
//   * integer SUM wraps in two's complement like the u64 atomicAdd of
//     src/cuda/atomics/atomics.cuh:22-126.
// Accumulators live in 64-bit lanes: signed ints widen to int64, unsigned to
// uint64, float32/float64 to double (exact), so MIN/MAX narrow back exactly.
#pragma once

#include "gx_core.cuh"

namespace gx {

constexpr int MAX_VCOLS = 8;   // distinct value columns read by one kernel
constexpr int MAX_ACCS = 16;   // accumulators per group (excluding COUNT)

enum acc_op : int { OP_SUM = 0, OP_MIN = 1, OP_MAX = 2, OP_ANY = 3 };

// Kernel-side description of what to aggregate (passed by value).
struct agg_desc {
    int n_cols = 0;
    const void* col_ptr[MAX_VCOLS] = {};
    int col_width[MAX_VCOLS] = {};
    int col_kind[MAX_VCOLS] = {};  // vkind
    int n_acc = 0;
    int acc_op[MAX_ACCS] = {};
    int acc_col[MAX_ACCS] = {};    // index into col_*
    int acc_kind[MAX_ACCS] = {};   // vkind of the lane
    int has_count = 0;
    // Record layout of a group: word 0 = key bits, word 1 = count (if any),
    // then one word per accumulator; rec_words is padded to a power of two.
    int count_word = -1;
    int acc_word0 = 1;
    int rec_words = 2;
    // The same accumulators grouped by update class, so hot loops run one
    // branch-free body per class: integer SUM, float SUM, MIN, MAX, ANY.
    int n_cls[5] = {};
    unsigned char cls_acc[5][MAX_ACCS] = {};
    unsigned char cls_col[5][MAX_ACCS] = {};
    unsigned char cls_kind[5][MAX_ACCS] = {};
};
enum acc_class : int { CL_ISUM = 0, CL_FSUM = 1, CL_MIN = 2, CL_MAX = 3, CL_ANY = 4 };

// Host-side plan: agg_desc + how to emit the reference's output columns.
struct out_spec {
    enum kind_t { ACC = 0, COUNT = 1, AVG = 2 } kind = ACC;
    int acc = -1;         // accumulator index (ACC / AVG numerator)
    int out_type = GX_EMPTY;
    int in_type = GX_EMPTY;
};

struct agg_plan {
    agg_desc d;
    std::vector<out_spec> outs;  // request order (+ trailing COUNT if agg_count)
    std::vector<int> col_types;  // input type of each distinct column
    std::vector<int> col_src;    // source column index in the value table
    int64_t value_bytes_per_row = 0;  // distinct value bytes read per row
};

int agg_output_type(int agg_kind, int input_type);

// Build the plan from the reference-shaped request list.
agg_plan make_agg_plan(const gx_table_view* val, const gx_agg_request* req, int nreq,
                       bool agg_count_hint);

// Identity words for the accumulators (host).
uint64_t acc_identity(int op, int kind);

// Records -> output table.  `recs` holds `nrec` records of d.rec_words words.
// When `compact` is true, records whose key word equals `empty_key` are
// skipped, except the record at index `sentinel_rec` (the group of the key
// whose bits equal the empty marker), which is emitted when the device flag
// `*sentinel_flag` is non-zero.
void emit_groupby_output(const agg_plan& p, const uint64_t* recs, int64_t nrec, bool compact,
                         uint64_t empty_key, int64_t sentinel_rec, const int* sentinel_flag,
                         int key_type, int64_t out_capacity, cudaStream_t s, gx_table* out);

#ifdef __CUDACC__
namespace dev_ {

// Load element `i` of a column as a 64-bit lane value.
__device__ __forceinline__ uint64_t load_lane(const void* base, int width, int kind, int64_t i) {
    switch (width) {
        case 8: return __ldg(static_cast<const unsigned long long*>(base) + i);
        case 4: {
            uint32_t b = __ldg(static_cast<const unsigned int*>(base) + i);
            if (kind == VK_F) return (uint64_t)__double_as_longlong((double)__uint_as_float(b));
            if (kind == VK_I) return (uint64_t)(int64_t)(int32_t)b;
            return (uint64_t)b;
        }
        case 2: {
            uint16_t b = static_cast<const uint16_t*>(base)[i];
            if (kind == VK_I) return (uint64_t)(int64_t)(int16_t)b;
            return (uint64_t)b;
        }
        default: {
            uint8_t b = static_cast<const uint8_t*>(base)[i];
            if (kind == VK_I) return (uint64_t)(int64_t)(int8_t)b;
            return (uint64_t)b;
        }
    }
}

// v[c] for a runtime c without dynamic register indexing.
template <int N>
__device__ __forceinline__ uint64_t pick(const uint64_t (&v)[N], int c) {
    uint64_t x = v[0];
#pragma unroll
    for (int k = 1; k < N; ++k)
        if (c == k) x = v[k];
    return x;
}

// Widen raw 32-bit bits according to kind (for vectorised loads).
__device__ __forceinline__ uint64_t widen32(uint32_t b, int kind) {
    if (kind == VK_F) return (uint64_t)__double_as_longlong((double)__uint_as_float(b));
    if (kind == VK_I) return (uint64_t)(int64_t)(int32_t)b;
    return (uint64_t)b;
}

// Combine v into *p (global or shared generic address).  Integer SUM is a
// u64 add (wraps), float SUM a double add; MIN/MAX on doubles use the
// sign-split integer atomics (same idea as src/cuda/atomics/atomics.cuh).
__device__ __forceinline__ void acc_atomic(uint64_t* p, int op, int kind, uint64_t v) {
    switch (op) {
        case OP_SUM:
            if (kind == VK_F) atomicAdd(reinterpret_cast<double*>(p), __longlong_as_double((long long)v));
            else atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
            break;
        case OP_MIN:
            if (kind == VK_I) atomicMin(reinterpret_cast<long long*>(p), (long long)v);
            else if (kind == VK_U) atomicMin(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
            else {
                double d = __longlong_as_double((long long)v);
                if (d != d) break;  // NaN does not participate
                if (!((long long)v < 0)) atomicMin(reinterpret_cast<long long*>(p), (long long)v);
                else atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
            }
            break;
        case OP_MAX:
            if (kind == VK_I) atomicMax(reinterpret_cast<long long*>(p), (long long)v);
            else if (kind == VK_U) atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
            else {
                double d = __longlong_as_double((long long)v);
                if (d != d) break;
                if (!((long long)v < 0)) atomicMax(reinterpret_cast<long long*>(p), (long long)v);
                else atomicMin(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
            }
            break;
        default:  // ANY: any row's value
            *reinterpret_cast<volatile unsigned long long*>(p) = v;
            break;
    }
}

// Would v move the MIN / MAX accumulator `cur`?  Doubles compare in the
// order the sign-split integer atomics of acc_atomic impose (-0.0 below
// +0.0); NaN never improves, as NaN never participates.
__device__ __forceinline__ bool improves(int op, int kind, uint64_t v, uint64_t cur) {
    if (kind == VK_I) return op == OP_MIN ? (long long)v < (long long)cur : (long long)v > (long long)cur;
    if (kind == VK_U) return op == OP_MIN ? v < cur : v > cur;
    const double d = __longlong_as_double((long long)v);
    if (d != d) return false;
    const uint64_t a = v ^ (((long long)v >> 63) ? ~0ull : 0x8000000000000000ull);
    const uint64_t b = cur ^ (((long long)cur >> 63) ? ~0ull : 0x8000000000000000ull);
    return op == OP_MIN ? a < b : a > b;
}

// Shared-memory update tuned for B200, where only 32-bit integer shared
// atomics are native (64-bit ones are compare-and-swap loops, 5-30x slower):
//   * integer SUM: two 32-bit adds — the low word's carry (detected from
//     the returned old value) goes into the high word, so the 64-bit result
//     is exact and wraps like the reference's u64 atomicAdd;
//   * MIN / MAX: a plain read first; the 64-bit atomic runs only when the
//     value would change the extreme (rare after the first rows of a group);
//   * float SUM: the native double atomicAdd;  ANY: a plain store.
__device__ __forceinline__ void acc_shared(uint64_t* p, int op, int kind, uint64_t v) {
    switch (op) {
        case OP_SUM:
            if (kind == VK_F) {
                atomicAdd(reinterpret_cast<double*>(p), __longlong_as_double((long long)v));
            } else {
                unsigned* w = reinterpret_cast<unsigned*>(p);
                unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
                unsigned old = atomicAdd(w, lo);
                hi += (old + lo) < old ? 1u : 0u;
                if (hi) atomicAdd(w + 1, hi);
            }
            break;
        case OP_MIN:
        case OP_MAX:
            if (improves(op, kind, v, *reinterpret_cast<volatile uint64_t*>(p))) acc_atomic(p, op, kind, v);
            break;
        default:
            *reinterpret_cast<volatile unsigned long long*>(p) = v;
            break;
    }
}

// Identity word of an accumulator.
__device__ __forceinline__ uint64_t acc_ident(int op, int kind) {
    if (op == OP_MIN) return kind == VK_I ? 0x7FFFFFFFFFFFFFFFull : (kind == VK_U ? ~0ull : 0x7FF0000000000000ull);
    if (op == OP_MAX) return kind == VK_I ? 0x8000000000000000ull : (kind == VK_U ? 0ull : 0xFFF0000000000000ull);
    return 0ull;
}

// Non-atomic combine of two lane values (register-level reductions).
__device__ __forceinline__ uint64_t acc_combine(int op, int kind, uint64_t a, uint64_t b) {
    switch (op) {
        case OP_SUM:
            if (kind == VK_F)
                return (uint64_t)__double_as_longlong(__longlong_as_double((long long)a) +
                                                      __longlong_as_double((long long)b));
            return a + b;
        case OP_MIN:
            if (kind == VK_I) return (long long)a < (long long)b ? a : b;
            if (kind == VK_U) return a < b ? a : b;
            {
                double x = __longlong_as_double((long long)a), y = __longlong_as_double((long long)b);
                if (y != y) return a;
                if (x != x) return b;
                return y < x ? b : a;
            }
        case OP_MAX:
            if (kind == VK_I) return (long long)a > (long long)b ? a : b;
            if (kind == VK_U) return a > b ? a : b;
            {
                double x = __longlong_as_double((long long)a), y = __longlong_as_double((long long)b);
                if (y != y) return a;
                if (x != x) return b;
                return y > x ? b : a;
            }
        default:
            return b;
    }
}

// One row's update of a shared-memory table: accumulator a of `slot` lives
// at acc[a * stride + slot].  Loops per update class (see agg_desc), each
// with a fixed body; see acc_shared for the per-class atomics used.
template <int NV>
__device__ __forceinline__ void shared_row_update(uint64_t* acc, size_t stride, int slot, const agg_desc& d,
                                                  const uint64_t (&v)[NV]) {
    for (int j = 0; j < d.n_cls[CL_ISUM]; ++j) {
        uint64_t x = pick(v, d.cls_col[CL_ISUM][j]);
        unsigned* w = reinterpret_cast<unsigned*>(acc + d.cls_acc[CL_ISUM][j] * stride + slot);
        unsigned lo = (unsigned)x, hi = (unsigned)(x >> 32);
        unsigned old = atomicAdd(w, lo);
        hi += (old + lo) < old ? 1u : 0u;
        if (hi) atomicAdd(w + 1, hi);
    }
    for (int j = 0; j < d.n_cls[CL_FSUM]; ++j) {
        double x = __longlong_as_double((long long)pick(v, d.cls_col[CL_FSUM][j]));
        atomicAdd(reinterpret_cast<double*>(acc + d.cls_acc[CL_FSUM][j] * stride + slot), x);
    }
    for (int j = 0; j < d.n_cls[CL_MIN]; ++j)
        acc_shared(acc + d.cls_acc[CL_MIN][j] * stride + slot, OP_MIN, d.cls_kind[CL_MIN][j],
                   pick(v, d.cls_col[CL_MIN][j]));
    for (int j = 0; j < d.n_cls[CL_MAX]; ++j)
        acc_shared(acc + d.cls_acc[CL_MAX][j] * stride + slot, OP_MAX, d.cls_kind[CL_MAX][j],
                   pick(v, d.cls_col[CL_MAX][j]));
    for (int j = 0; j < d.n_cls[CL_ANY]; ++j)
        *reinterpret_cast<volatile unsigned long long*>(acc + d.cls_acc[CL_ANY][j] * stride + slot) =
            pick(v, d.cls_col[CL_ANY][j]);
}

}  // namespace dev_
#endif

}  // namespace gx
