// gx_agg.cu — request rewriting and record -> column emission shared by all
// group-by variants (see gx_agg.cuh for the semantics followed).
#include <algorithm>
#include <cmath>
#include <limits>

#include "gx_agg.cuh"

namespace gx {

int agg_output_type(int agg_kind, int t) {
    if (agg_kind == GX_AGG_COUNT_ALL) return GX_INT64;
    if (agg_kind == GX_AGG_AVG) return GX_FLOAT64;
    if (agg_kind == GX_AGG_SUM) {
        switch (t) {
            case GX_INT8: case GX_INT16: case GX_INT32: case GX_INT64: return GX_INT64;
            case GX_UINT8: case GX_UINT16: case GX_UINT32: case GX_UINT64: return GX_UINT64;
            case GX_FLOAT32: return GX_FLOAT32;
            case GX_FLOAT64: return GX_FLOAT64;
            default: return GX_EMPTY;
        }
    }
    if (agg_kind == GX_AGG_MIN || agg_kind == GX_AGG_MAX || agg_kind == GX_AGG_ANY)
        return is_numeric(t) && t != GX_BOOL8 ? t : GX_EMPTY;
    return GX_EMPTY;
}

uint64_t acc_identity(int op, int kind) {
    switch (op) {
        case OP_SUM: return 0;
        case OP_MIN:
            if (kind == VK_I) return (uint64_t)std::numeric_limits<int64_t>::max();
            if (kind == VK_U) return ~uint64_t(0);
            return 0x7FF0000000000000ull;  // +inf
        case OP_MAX:
            if (kind == VK_I) return (uint64_t)std::numeric_limits<int64_t>::min();
            if (kind == VK_U) return 0;
            return 0xFFF0000000000000ull;  // -inf
        default: return 0;
    }
}

agg_plan make_agg_plan(const gx_table_view* val, const gx_agg_request* req, int nreq,
                       bool agg_count_hint) {
    agg_plan p;
    require(nreq >= 0 && (nreq == 0 || req != nullptr), "bad aggregation request list");
    int64_t nvals = val ? val->num_columns : 0;
    auto col_slot = [&](int64_t ci) -> int {
        require(ci >= 0 && ci < nvals, "aggregation column index " + std::to_string(ci) +
                                           " out of range (value table has " +
                                           std::to_string(nvals) + " columns)");
        for (size_t k = 0; k < p.col_src.size(); ++k)
            if (p.col_src[k] == (int)ci) return (int)k;
        const gx_column_view& v = val->columns[ci];
        require(is_numeric(v.type) && v.type != GX_BOOL8,
                "aggregation over unsupported column type " + type_name(v.type));
        require((int)p.col_src.size() < MAX_VCOLS, "too many distinct value columns");
        int k = (int)p.col_src.size();
        col c = resolve(v);
        p.col_src.push_back((int)ci);
        p.col_types.push_back(v.type);
        p.d.col_ptr[k] = c.data;
        p.d.col_width[k] = size_of(v.type);
        p.d.col_kind[k] = vkind_of(v.type);
        p.value_bytes_per_row += size_of(v.type);
        p.d.n_cols = k + 1;
        return k;
    };
    auto acc_slot = [&](int op, int slot) -> int {
        for (int a = 0; a < p.d.n_acc; ++a)
            if (p.d.acc_op[a] == op && p.d.acc_col[a] == slot) return a;
        require(p.d.n_acc < MAX_ACCS, "too many aggregations");
        int a = p.d.n_acc++;
        p.d.acc_op[a] = op;
        p.d.acc_col[a] = slot;
        p.d.acc_kind[a] = p.d.col_kind[slot];
        return a;
    };
    bool need_count = agg_count_hint;
    for (int r = 0; r < nreq; ++r) {
        out_spec o;
        switch (req[r].agg_kind) {
            case GX_AGG_SUM: case GX_AGG_MIN: case GX_AGG_MAX: case GX_AGG_ANY: {
                int s = col_slot(req[r].column_index);
                int op = req[r].agg_kind == GX_AGG_SUM ? OP_SUM
                       : req[r].agg_kind == GX_AGG_MIN ? OP_MIN
                       : req[r].agg_kind == GX_AGG_MAX ? OP_MAX : OP_ANY;
                o.kind = out_spec::ACC;
                o.acc = acc_slot(op, s);
                o.in_type = p.col_types[s];
                o.out_type = agg_output_type(req[r].agg_kind, o.in_type);
                break;
            }
            case GX_AGG_AVG: {
                int s = col_slot(req[r].column_index);
                o.kind = out_spec::AVG;
                o.acc = acc_slot(OP_SUM, s);
                o.in_type = p.col_types[s];
                o.out_type = GX_FLOAT64;
                need_count = true;
                break;
            }
            case GX_AGG_COUNT_ALL:
                o.kind = out_spec::COUNT;
                o.out_type = GX_INT64;
                need_count = true;
                break;
            default:
                fail(GX_EINVAL, "Unsupported aggregation function");
        }
        require(o.out_type != GX_EMPTY, "unsupported aggregation output type");
        p.outs.push_back(o);
    }
    if (agg_count_hint) {
        out_spec o;
        o.kind = out_spec::COUNT;
        o.out_type = GX_INT64;
        p.outs.push_back(o);
    }
    for (int a = 0; a < p.d.n_acc; ++a) {
        int op = p.d.acc_op[a], kind = p.d.acc_kind[a];
        int cl = op == OP_SUM ? (kind == VK_F ? CL_FSUM : CL_ISUM) : op == OP_MIN ? CL_MIN : op == OP_MAX ? CL_MAX : CL_ANY;
        int j = p.d.n_cls[cl]++;
        p.d.cls_acc[cl][j] = (unsigned char)a;
        p.d.cls_col[cl][j] = (unsigned char)p.d.acc_col[a];
        p.d.cls_kind[cl][j] = (unsigned char)kind;
    }
    p.d.has_count = need_count ? 1 : 0;
    p.d.count_word = need_count ? 1 : -1;
    p.d.acc_word0 = 1 + (need_count ? 1 : 0);
    int words = p.d.acc_word0 + p.d.n_acc;
    int padded = 1;
    while (padded < words) padded <<= 1;
    p.d.rec_words = padded;
    return p;
}

namespace {

constexpr int EMIT_NT = 256;

struct emit_args {
    const uint64_t* recs;
    int64_t nrec;
    int rec_words;
    int compact;
    uint64_t empty_key;
    int64_t sentinel_rec;
    const int* sentinel_flag;
    int key_width;
    void* key_out;
    int n_out;
    void* out_ptr[MAX_ACCS + 4];
    int out_kind[MAX_ACCS + 4];  // out_spec::kind_t
    int out_word[MAX_ACCS + 4];  // word of the accumulator (ACC / AVG)
    int out_type[MAX_ACCS + 4];
    int out_lane_kind[MAX_ACCS + 4];
    int count_word;
};

__device__ __forceinline__ bool rec_live(const emit_args& a, int64_t r) {
    if (!a.compact) return true;
    if (r == a.sentinel_rec) return a.sentinel_flag != nullptr && *a.sentinel_flag != 0;
    return a.recs[r * a.rec_words] != a.empty_key;
}

__global__ void __launch_bounds__(EMIT_NT) k_emit_count(emit_args a, int64_t* __restrict__ blk) {
    int64_t r = blockIdx.x * (int64_t)EMIT_NT + threadIdx.x;
    int live = (r < a.nrec && rec_live(a, r)) ? 1 : 0;
    int c = __syncthreads_count(live);
    if (threadIdx.x == 0) blk[blockIdx.x] = c;
}

__device__ __forceinline__ void store_typed(void* base, int type, int64_t i, uint64_t lane, int lane_kind) {
    switch (type) {
        case GX_INT8: static_cast<int8_t*>(base)[i] = (int8_t)(int64_t)lane; break;
        case GX_UINT8: static_cast<uint8_t*>(base)[i] = (uint8_t)lane; break;
        case GX_INT16: static_cast<int16_t*>(base)[i] = (int16_t)(int64_t)lane; break;
        case GX_UINT16: static_cast<uint16_t*>(base)[i] = (uint16_t)lane; break;
        case GX_INT32: static_cast<int32_t*>(base)[i] = (int32_t)(int64_t)lane; break;
        case GX_UINT32: static_cast<uint32_t*>(base)[i] = (uint32_t)lane; break;
        case GX_FLOAT32:
            static_cast<float*>(base)[i] = (float)__longlong_as_double((long long)lane);
            break;
        default: static_cast<uint64_t*>(base)[i] = lane; break;  // 8-byte types
    }
}

__global__ void __launch_bounds__(EMIT_NT) k_emit_write(emit_args a, const int64_t* __restrict__ blk_off) {
    __shared__ int64_t sm[EMIT_NT / 32 + 1];
    int64_t r = blockIdx.x * (int64_t)EMIT_NT + threadIdx.x;
    bool live = r < a.nrec && rec_live(a, r);
    int64_t total;
    // Dense records (no compaction) sit at their own index.
    const int64_t base = a.compact ? blk_off[blockIdx.x] : blockIdx.x * (int64_t)EMIT_NT;
    int64_t pos = dev_::block_exclusive_sum<EMIT_NT, int64_t>(live ? 1 : 0, sm, &total) + base;
    if (!live) return;
    const uint64_t* rec = a.recs + r * a.rec_words;
    uint64_t kb = rec[0];
    switch (a.key_width) {
        case 8: static_cast<uint64_t*>(a.key_out)[pos] = kb; break;
        case 4: static_cast<uint32_t*>(a.key_out)[pos] = (uint32_t)kb; break;
        case 2: static_cast<uint16_t*>(a.key_out)[pos] = (uint16_t)kb; break;
        default: static_cast<uint8_t*>(a.key_out)[pos] = (uint8_t)kb; break;
    }
    for (int o = 0; o < a.n_out; ++o) {
        if (a.out_kind[o] == 1) {  // COUNT
            static_cast<int64_t*>(a.out_ptr[o])[pos] = (int64_t)rec[a.count_word];
        } else if (a.out_kind[o] == 2) {  // AVG = SUM / COUNT in double
            uint64_t s = rec[a.out_word[o]];
            double num;
            if (a.out_lane_kind[o] == VK_F) num = __longlong_as_double((long long)s);
            else if (a.out_lane_kind[o] == VK_I) num = (double)(long long)s;
            else num = (double)(unsigned long long)s;
            static_cast<double*>(a.out_ptr[o])[pos] = num / (double)(long long)rec[a.count_word];
        } else {
            store_typed(a.out_ptr[o], a.out_type[o], pos, rec[a.out_word[o]], a.out_lane_kind[o]);
        }
    }
}

}  // namespace

void emit_groupby_output(const agg_plan& p, const uint64_t* recs, int64_t nrec, bool compact,
                         uint64_t empty_key, int64_t sentinel_rec, const int* sentinel_flag,
                         int key_type, int64_t out_capacity, cudaStream_t s, gx_table* out) {
    emit_args a;
    std::memset(&a, 0, sizeof(a));
    a.recs = recs;
    a.nrec = nrec;
    a.rec_words = p.d.rec_words;
    a.compact = compact ? 1 : 0;
    a.empty_key = empty_key;
    a.sentinel_rec = sentinel_rec;
    a.sentinel_flag = sentinel_flag;
    a.key_width = size_of(key_type);
    a.count_word = p.d.count_word;
    a.n_out = (int)p.outs.size();
    int64_t nblk = ceil_div(nrec > 0 ? nrec : 1, EMIT_NT);
    dbuf blk(nblk * sizeof(int64_t), s), off((nblk + 1) * sizeof(int64_t), s);
    int64_t groups = nrec;
    if (compact) {
        k_emit_count<<<(unsigned)nblk, EMIT_NT, 0, s>>>(a, blk.get<int64_t>());
        GX_LAUNCHED();
        exclusive_scan_i64(blk.get<int64_t>(), off.get<int64_t>(), nblk, s);
        groups = read_scalar(off.get<int64_t>() + nblk, s);
    }
    int64_t cap = std::max<int64_t>(groups, std::min<int64_t>(out_capacity, groups));
    out->cols.clear();
    out->cols.push_back(make_col(key_type, groups, s, cap));
    a.key_out = out->cols.back().buf.get();
    for (size_t o = 0; o < p.outs.size(); ++o) {
        const out_spec& os = p.outs[o];
        out->cols.push_back(make_col(os.out_type, groups, s, cap));
        a.out_ptr[o] = out->cols.back().buf.get();
        a.out_kind[o] = (int)os.kind;
        a.out_type[o] = os.out_type;
        a.out_word[o] = os.acc >= 0 ? p.d.acc_word0 + os.acc : 0;
        a.out_lane_kind[o] = os.acc >= 0 ? p.d.acc_kind[os.acc] : VK_I;
    }
    if (groups > 0) {
        k_emit_write<<<(unsigned)nblk, EMIT_NT, 0, s>>>(a, off.get<int64_t>());
        GX_LAUNCHED();
    }
}

}  // namespace gx
