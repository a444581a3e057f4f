// gx_join.h — internal interfaces shared by the join translation units
// (gx_join.cu: sort-based and dense plans; gx_join_hash.cu: hash and
// partitioned-hash plans).
#pragma once

#include "gx_groupby.h"

namespace gx {

constexpr int MAX_PAY = 8;

struct join_inputs {
    col lkey, rkey;
    std::vector<col> lpay, rpay;
};

// Where each output column of a join comes from.
struct join_out {
    // Output columns: key, then the build side's payloads and the probe
    // side's, in the caller's left/right order.
    void* key;              // may be null (row-id form)
    int key_width;
    int n_pay;              // total payload outputs
    void* out[2 * MAX_PAY + 2];
    int width[2 * MAX_PAY + 2];
    // source: 0 = build run value (sorted payload / row id), 1 = build column
    // gathered by build row id, 2 = probe column at probe row, 3 = build row id,
    // 4 = probe row id
    int src[2 * MAX_PAY + 2];
    const void* col[2 * MAX_PAY + 2];
};

// Allocates the output columns of a join with `total` rows (capacity `cap`
// rows when cap >= 0) and describes their sources: [key, left payloads..,
// right payloads..], or the (left_rowid, right_rowid) pair when
// rowids_only.  `dense` (or a plan that matches by row ids) reads build
// payloads by build row id.
join_out make_outputs(const join_inputs& in, bool build_left, bool rowids_only, bool pay_in_run, bool dense,
                      int64_t total, cudaStream_t s, gx_table* out, int64_t cap = -1);

// Hash join (join_algo HASH) and partitioned hash join (join_algo
// PARTITION); gx_join_hash.cu.
void hash_join(const join_inputs& in, const gx_join_hint& hint, bool rowids_only, cudaStream_t s, gx_table* out);
void partition_hash_join(const join_inputs& in, const gx_join_hint& hint, bool rowids_only, cudaStream_t s,
                         gx_table* out);

#ifdef __CUDACC__
__device__ __forceinline__ uint64_t ld_w(const void* p, int w, int64_t i) {
    switch (w) {
        case 8: return __ldg(static_cast<const unsigned long long*>(p) + i);
        case 4: return __ldg(static_cast<const unsigned*>(p) + i);
        case 2: return static_cast<const uint16_t*>(p)[i];
        default: return static_cast<const uint8_t*>(p)[i];
    }
}
// Join outputs are written once: 4/8-byte stores use the streaming hint.
__device__ __forceinline__ void st_w(void* p, int w, int64_t i, uint64_t v) {
    switch (w) {
        case 8: __stcs(static_cast<unsigned long long*>(p) + i, (unsigned long long)v); break;
        case 4: __stcs(static_cast<unsigned*>(p) + i, (unsigned)v); break;
        case 2: static_cast<uint16_t*>(p)[i] = (uint16_t)v; break;
        default: static_cast<uint8_t*>(p)[i] = (uint8_t)v; break;
    }
}
// One matched pair's output row: sources 1 = build column at the build row,
// 2 = probe column at the probe row, 3 = build row id, 4 = probe row id; the
// key column takes the probe row's key.
__device__ __forceinline__ void write_pair(const join_out& o, const void* pkeys, int64_t pos, int64_t brow,
                                           int64_t prow) {
    if (o.key) st_w(o.key, o.key_width, pos, ld_w(pkeys, o.key_width, prow));
    for (int c = 0; c < o.n_pay; ++c) {
        uint64_t v;
        switch (o.src[c]) {
            case 1: v = ld_w(o.col[c], o.width[c], brow); break;
            case 2: v = ld_w(o.col[c], o.width[c], prow); break;
            case 3: v = (uint64_t)brow; break;
            default: v = (uint64_t)prow; break;
        }
        st_w(o.out[c], o.width[c], pos, v);
    }
}
#endif

}  // namespace gx
