// gx_select.cu — filter: predicate -> BOOL8 mask -> order-preserving
// compaction, and the fused form that evaluates the predicate while
// compacting.
//
// Replaces gamax::select::select_to_bitmask / select (src/cuda/operators/
// select/select.hpp:15-64, select.cu:19-60) for predicates that are a
// conjunction or disjunction of comparisons of a column with literals, and
// gamax::util::device::compact / count_nonzero (src/cuda/utils/transform.hpp:
// 34-48, transform.cu:74-95,147-205: cub::DeviceSelect::Flagged per column
// plus a thrust reduction of the mask).  The reference's general expression
// trees (expr/expr_fast.hpp) are outside this library.
//
// B200 design: rows are taken in 4096-row tiles (256 threads x 16 rows, the
// rows of a warp contiguous).  A count kernel evaluates the predicate (or
// reads the mask) and writes each tile's kept-row count; an exclusive scan
// places the tiles; a write kernel evaluates again, ranks the kept rows
// inside the tile with warp ballots and a block scan, and writes every
// column's kept values to consecutive positions — one pass over the input
// per kernel, kept rows in input order (the order cub::DeviceSelect keeps).
#include "gx_groupby.h"

namespace gx {
namespace {

constexpr int SL_NT = 256;
constexpr int SL_IPT = 16;
constexpr int SL_TILE = SL_NT * SL_IPT;
constexpr int MAX_PRED = 8;
constexpr int MAX_SEL_COLS = 32;

struct pred_dev {
    int n;
    int combine;  // 0 = AND, 1 = OR
    const void* data[MAX_PRED];
    int width[MAX_PRED];
    int kind[MAX_PRED];
    int op[MAX_PRED];
    int64_t lo_i[MAX_PRED], hi_i[MAX_PRED];
    double lo_f[MAX_PRED], hi_f[MAX_PRED];
    const uint8_t* mask;  // when non-null: keep = mask[row] != 0, predicates unused
};

struct sel_cols {
    int n;
    const void* in[MAX_SEL_COLS];
    void* out[MAX_SEL_COLS];
    int width[MAX_SEL_COLS];
};

template <class T>
__device__ __forceinline__ bool cmp(int op, T x, T lo, T hi) {
    switch (op) {
        case GX_CMP_LT: return x < lo;
        case GX_CMP_LE: return x <= lo;
        case GX_CMP_GT: return x > lo;
        case GX_CMP_GE: return x >= lo;
        case GX_CMP_EQ: return x == lo;
        case GX_CMP_NE: return x != lo;
        default: return x >= lo && x < hi;  // BETWEEN: lo <= x < hi
    }
}

__device__ __forceinline__ bool eval_one(const pred_dev& p, int j, int64_t i) {
    const void* d = p.data[j];
    const int op = p.op[j];
    if (p.kind[j] == VK_F) {
        const double x = p.width[j] == 4 ? (double)static_cast<const float*>(d)[i] : static_cast<const double*>(d)[i];
        return cmp<double>(op, x, p.lo_f[j], p.hi_f[j]);
    }
    if (p.kind[j] == VK_U) {
        uint64_t x;
        switch (p.width[j]) {
            case 1: x = static_cast<const uint8_t*>(d)[i]; break;
            case 2: x = static_cast<const uint16_t*>(d)[i]; break;
            case 4: x = static_cast<const uint32_t*>(d)[i]; break;
            default: x = static_cast<const uint64_t*>(d)[i]; break;
        }
        return cmp<uint64_t>(op, x, (uint64_t)p.lo_i[j], (uint64_t)p.hi_i[j]);
    }
    int64_t x;
    switch (p.width[j]) {
        case 1: x = static_cast<const int8_t*>(d)[i]; break;
        case 2: x = static_cast<const int16_t*>(d)[i]; break;
        case 4: x = static_cast<const int32_t*>(d)[i]; break;
        default: x = static_cast<const int64_t*>(d)[i]; break;
    }
    return cmp<int64_t>(op, x, p.lo_i[j], p.hi_i[j]);
}

__device__ __forceinline__ bool keep_row(const pred_dev& p, int64_t i) {
    if (p.mask) return p.mask[i] != 0;
    if (p.combine == 0) {
        for (int j = 0; j < p.n; ++j)
            if (!eval_one(p, j, i)) return false;
        return true;
    }
    for (int j = 0; j < p.n; ++j)
        if (eval_one(p, j, i)) return true;
    return false;
}

__global__ void k_sel_mask(pred_dev p, int64_t n, uint8_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = keep_row(p, i) ? 1 : 0;
}

// Row (k, lane) of warp w in tile t: t*TILE + w*32*IPT + k*32 + lane.
__global__ void __launch_bounds__(SL_NT) k_sel_count(pred_dev p, int64_t n, int64_t* __restrict__ tile_cnt) {
    __shared__ int sm[SL_NT / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row0 = blockIdx.x * (int64_t)SL_TILE + warp * 32 * SL_IPT + lane;
    int c = 0;
#pragma unroll 4
    for (int k = 0; k < SL_IPT; ++k) {
        const int64_t i = row0 + k * 32;
        c += i < n && keep_row(p, i);
    }
    c = dev_::warp_sum(c);
    if (lane == 0) sm[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < SL_NT / 32; ++w) t += sm[w];
        tile_cnt[blockIdx.x] = t;
    }
}

__device__ __forceinline__ void copy_elem(const sel_cols& c, int j, int64_t src, int64_t dst) {
    switch (c.width[j]) {
        case 1: static_cast<uint8_t*>(c.out[j])[dst] = static_cast<const uint8_t*>(c.in[j])[src]; break;
        case 2: static_cast<uint16_t*>(c.out[j])[dst] = static_cast<const uint16_t*>(c.in[j])[src]; break;
        case 4: static_cast<uint32_t*>(c.out[j])[dst] = __ldg(static_cast<const uint32_t*>(c.in[j]) + src); break;
        default: static_cast<uint64_t*>(c.out[j])[dst] = __ldg(static_cast<const unsigned long long*>(c.in[j]) + src); break;
    }
}

__global__ void __launch_bounds__(SL_NT) k_sel_write(pred_dev p, int64_t n, const int64_t* __restrict__ tile_off,
                                                      sel_cols c) {
    __shared__ int64_t sm[SL_NT / 32 + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row0 = blockIdx.x * (int64_t)SL_TILE + warp * 32 * SL_IPT + lane;
    unsigned keep = 0;  // bit k: row (k, lane) is kept
#pragma unroll 4
    for (int k = 0; k < SL_IPT; ++k) {
        const int64_t i = row0 + k * 32;
        if (i < n && keep_row(p, i)) keep |= 1u << k;
    }
    const int64_t mine = __popc(keep);
    const int64_t wtot = dev_::warp_sum(mine);
    int64_t total;
    int64_t base = dev_::block_exclusive_sum<SL_NT, int64_t>(lane == 0 ? wtot : 0, sm, &total);
    base = __shfl_sync(0xffffffffu, base, 0) + tile_off[blockIdx.x];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll 4
    for (int k = 0; k < SL_IPT; ++k) {
        const bool kept = (keep >> k) & 1u;
        const unsigned bal = __ballot_sync(0xffffffffu, kept);
        if (kept) {
            const int64_t dst = base + __popc(bal & lt);
            for (int j = 0; j < c.n; ++j) copy_elem(c, j, row0 + k * 32, dst);
        }
        base += __popc(bal);
    }
}

pred_dev make_preds(const gx_table_view* t, const gx_predicate* preds, int n, int combine) {
    require(t != nullptr, "select: null table");
    require(n >= 1 && n <= MAX_PRED, "select: 1 to " + std::to_string(MAX_PRED) + " predicates supported");
    require(preds != nullptr, "select: null predicates");
    require(combine == GX_COMBINE_AND || combine == GX_COMBINE_OR, "select: combine must be AND or OR");
    pred_dev p;
    std::memset(&p, 0, sizeof(p));
    p.n = n;
    p.combine = combine;
    for (int j = 0; j < n; ++j) {
        const gx_predicate& q = preds[j];
        require(q.column_index >= 0 && q.column_index < t->num_columns, "select: predicate column out of range");
        const gx_column_view& v = t->columns[q.column_index];
        require(is_numeric(v.type), "select: predicates on " + type_name(v.type) + " columns are not supported");
        require(q.op >= GX_CMP_LT && q.op <= GX_CMP_BETWEEN, "select: unknown comparison");
        col c = resolve(v);
        p.data[j] = c.data;
        p.width[j] = size_of(v.type);
        p.kind[j] = vkind_of(v.type);
        p.op[j] = q.op;
        p.lo_i[j] = q.lo_i;
        p.hi_i[j] = q.hi_i;
        p.lo_f[j] = q.lo_f;
        p.hi_f[j] = q.hi_f;
    }
    return p;
}

int64_t table_rows(const gx_table_view* t) {
    const int64_t n = t->num_columns ? t->columns[0].size : 0;
    for (int64_t c = 0; c < t->num_columns; ++c)
        require(t->columns[c].size == n, "select: columns differ in length");
    return n;
}

// Count + scan + write of every column of `t` for the rows `p` keeps.
void compact_rows(const gx_table_view* t, const pred_dev& p, int64_t n, cudaStream_t s, gx_table* out) {
    require(t->num_columns <= MAX_SEL_COLS, "select: at most " + std::to_string(MAX_SEL_COLS) + " columns");
    for (int64_t c = 0; c < t->num_columns; ++c)
        if (!is_numeric(t->columns[c].type)) fail(GX_EUNSUPPORTED, "compact: STRING columns are not supported");
    const int64_t ntiles = ceil_div(std::max<int64_t>(n, 1), SL_TILE);
    dbuf tc((size_t)ntiles * 8, s), toff((size_t)(ntiles + 1) * 8, s);
    int64_t kept = 0;
    if (n > 0) {
        GX_PROF("select_count", s);
        k_sel_count<<<(unsigned)ntiles, SL_NT, 0, s>>>(p, n, tc.get<int64_t>());
        GX_LAUNCHED();
        exclusive_scan_i64(tc.get<int64_t>(), toff.get<int64_t>(), ntiles, s);
        kept = read_scalar(toff.get<int64_t>() + ntiles, s);
    }
    sel_cols sc;
    std::memset(&sc, 0, sizeof(sc));
    out->cols.clear();
    for (int64_t c = 0; c < t->num_columns; ++c) {
        out->cols.push_back(make_col(t->columns[c].type, kept, s));
        col in = resolve(t->columns[c]);
        sc.in[sc.n] = in.data;
        sc.out[sc.n] = out->cols.back().buf.get();
        sc.width[sc.n] = size_of(in.type);
        ++sc.n;
    }
    if (kept > 0) {
        GX_PROF("select_write", s);
        k_sel_write<<<(unsigned)ntiles, SL_NT, 0, s>>>(p, n, toff.get<int64_t>(), sc);
        GX_LAUNCHED();
    }
    GX_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

void select_to_bitmask(const gx_table_view* t, const gx_predicate* preds, int n, int combine, cudaStream_t s,
                       gx_column* mask) {
    pred_dev p = make_preds(t, preds, n, combine);
    const int64_t rows = table_rows(t);
    owned_col m = make_col(GX_BOOL8, rows, s);
    if (rows > 0) {
        k_sel_mask<<<grid_for(rows, 256, 8), 256, 0, s>>>(p, rows, m.buf.get<uint8_t>());
        GX_LAUNCHED();
    }
    GX_CUDA(cudaStreamSynchronize(s));
    *mask = to_gx_column(std::move(m));
}

void select_rows(const gx_table_view* t, const gx_predicate* preds, int n, int combine, cudaStream_t s,
                 gx_table* out) {
    pred_dev p = make_preds(t, preds, n, combine);
    compact_rows(t, p, table_rows(t), s, out);
}

void compact_by_mask(const gx_table_view* t, const gx_column_view& mask, cudaStream_t s, gx_table* out) {
    require(t != nullptr, "compact: null table");
    require(size_of(mask.type) == 1, "compact: the mask must be a BOOL8 / 1-byte column");
    const int64_t n = table_rows(t);
    require(mask.size == n || t->num_columns == 0, "compact: mask length differs from the table's rows");
    pred_dev p;
    std::memset(&p, 0, sizeof(p));
    p.mask = static_cast<const uint8_t*>(resolve(mask).data);
    compact_rows(t, p, t->num_columns ? n : 0, s, out);
}

int64_t count_nonzero(const gx_column_view& v, cudaStream_t s) {
    col c = resolve(v);
    require(is_numeric(c.type), "count_nonzero: numeric column required");
    if (c.n == 0) return 0;
    gx_predicate q;
    std::memset(&q, 0, sizeof(q));
    q.column_index = 0;
    q.op = GX_CMP_NE;
    gx_table_view t{&v, 1};
    pred_dev p = make_preds(&t, &q, 1, GX_COMBINE_AND);
    const int64_t ntiles = ceil_div(c.n, SL_TILE);
    dbuf tc((size_t)ntiles * 8, s), toff((size_t)(ntiles + 1) * 8, s);
    k_sel_count<<<(unsigned)ntiles, SL_NT, 0, s>>>(p, c.n, tc.get<int64_t>());
    GX_LAUNCHED();
    exclusive_scan_i64(tc.get<int64_t>(), toff.get<int64_t>(), ntiles, s);
    return read_scalar(toff.get<int64_t>() + ntiles, s);
}

}  // namespace gx
