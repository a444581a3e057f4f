// gx_batch.cu — many uneven string group-by pipelines in one launch.
//
// Each instance: dictionary-encode an ARROW string column (chars + int64
// offsets, src/cuda/string/string_column.hpp:22-90), keep rows with
// lo <= date < hi, and group the kept rows by the encoded key with SUM of an
// int64 fixed-point amount and COUNT.  The reference runs such a pipeline as
// separate operators per table (hash group-by on the STRING key after a
// select, src/cuda/operators/groupby/groupby_hash.cu:437-498,
// src/cuda/operators/select/select.hpp:15-64), with host syncs in between.
//
// Batched engine: one persistent kernel walks a work queue of row tiles of
// all instances (dynamic tile handout -> no tail effect from uneven sizes).
// A row finds or inserts its string in its instance's table — one 64-bit
// word per slot holding a 24-bit hash tag and the representative row, so a
// single CAS publishes a new entry and the bytes are compared against the
// representative row of the input, both read as 8-byte chunks of aligned
// words — gets the next dictionary code on insert, and adds its amount /
// count to the slot.  The date filter runs first: only kept rows are
// encoded (the output holds kept groups only), so the dictionary and its
// codes cover the kept rows' strings.  A finalize kernel
// writes the per-code results.  Both kernels and the resets are captured
// once into a CUDA graph and replayed.  Tile size and table load factor are
// chosen by timing the candidates on the batch.
//
// The plain engine (gx_batch_run_per_instance) runs the same work as one
// operator sequence per instance: string dictionary encode, filter with
// compaction, hash group-by on the codes.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "gx_groupby.h"

struct gx_batch_plan;

namespace gx {

void hash_groupby(const col& key, const agg_plan& p, gx_groupby_hint* hint, cudaStream_t s, gx_table* out);

namespace {

constexpr uint64_t ROW_MASK = (1ull << 40) - 1;

struct inst_dev {
    const char* chars;
    const int64_t* offsets;
    const int32_t* date;
    const int64_t* amount;
    int64_t rows;
    int32_t lo, hi;
    int64_t table_off;   // slot offset of this instance's table
    int64_t result_off;  // code offset of this instance's results
    int64_t clo, chi;    // byte range of chars the strings occupy: offsets[0], offsets[rows]
};

struct work_item {
    int32_t inst;
    int32_t pad;
    int64_t begin, end;
};

struct batch_dev {
    const inst_dev* inst;
    const work_item* work;
    int64_t n_work;
    unsigned long long* entries;  // [total slots]: tag << 40 | (row + 1); 0 = empty
    unsigned* code_of_slot;       // dictionary code of a slot, ~0u until published (see find_or_insert)
    unsigned long long* ks_key;   // [total codes][4]: first 32 bytes of the code's string, zero padded
    unsigned* ks_len;             // [total codes]: its length
    unsigned* slot_of_code;       // [total codes]: the code's slot in its instance's table
    unsigned long long* sum_slot;
    unsigned long long* cnt_slot;
    unsigned* dict_size;          // per instance
    unsigned long long* work_counter;
    int* overflow;
    uint32_t slots;               // per instance (power of two)
    uint32_t max_distinct;
    // finalize outputs (code order)
    long long* out_sum;
    long long* out_cnt;
    long long* out_first;
    long long* out_groups;        // per instance
};

// String bytes are read in 8-byte chunks assembled from aligned 8-byte words,
// so the consecutive strings of a warp's lanes come in coalesced words rather
// than one byte per load.  Every read stays inside the byte range
// [lo, hi) of `chars` that the column's strings occupy: an aligned word that
// reaches outside it is assembled from its in-range bytes.
struct char_span {
    const unsigned char* chars;
    int64_t lo, hi;
};

// An aligned word that reaches outside the span, assembled from its in-range
// bytes (kept out of line: it is the rare edge of a column).  The span comes
// in by value: a reference would make every caller keep its span in local
// memory.
__device__ __noinline__ uint64_t word_at_edge(const unsigned char* chars, int64_t lo, int64_t hi, int64_t a) {
    uint64_t w = 0;
    for (int k = 0; k < 8; ++k)
        if (a + k >= lo && a + k < hi) w |= (uint64_t)chars[a + k] << (8 * k);
    return w;
}

__device__ __forceinline__ uint64_t word_at(const char_span& c, int64_t a) {
    // a: position (relative to chars) of an 8-byte-aligned address
    if (a >= c.lo && a + 8 <= c.hi) return __ldg(reinterpret_cast<const unsigned long long*>(c.chars + a));
    return word_at_edge(c.chars, c.lo, c.hi, a);
}

// The first min(len, 32) bytes of the string at [pos, pos + len) as four
// little-endian 8-byte chunks (zero past the string), from at most five
// aligned words, in straight-line code.
__device__ __forceinline__ void load32(const char_span& c, int64_t pos, int64_t len, uint64_t (&ch)[4]) {
    const int mis = (int)(reinterpret_cast<uintptr_t>(c.chars + pos) & 7);
    const int64_t a = pos - mis;
    const int n = (int)(len < 32 ? len : 32);
    const int nw = (mis + n + 7) >> 3;
    uint64_t w[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) w[j] = j < nw ? word_at(c, a + 8 * j) : 0ull;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint64_t v = mis ? ((w[i] >> (8 * mis)) | (w[i + 1] << (64 - 8 * mis))) : w[i];
        const int rem = n - 8 * i;
        ch[i] = rem >= 8 ? v : (rem <= 0 ? 0ull : (v & ((1ull << (8 * rem)) - 1)));
    }
}

// Bytes [pos, pos + n) of the span, little-endian, n in 1..8, zero above.
__device__ __forceinline__ uint64_t chunk_at(const char_span& c, int64_t pos, int n) {
    const int mis = (int)(reinterpret_cast<uintptr_t>(c.chars + pos) & 7);
    const int64_t a = pos - mis;
    uint64_t v = word_at(c, a) >> (8 * mis);
    if (mis + n > 8) v |= word_at(c, a + 8) << (64 - 8 * mis);
    return n == 8 ? v : (v & ((1ull << (8 * n)) - 1));
}

// One multiply-xorshift round of the string hash over an 8-byte chunk.
__device__ __forceinline__ uint64_t hash_round(uint64_t h, uint64_t chunk) {
    h = (h ^ chunk) * 0xff51afd7ed558ccdull;
    return h ^ (h >> 32);
}

// Hash of the string whose first 32 bytes are in ch (load32) and whose
// remaining bytes, if any, follow at pos + 32.
__device__ __forceinline__ uint64_t str_hash_chunks(const char_span& c, int64_t pos, int64_t len,
                                                    const uint64_t (&ch)[4]) {
    uint64_t h = 0x9E3779B97F4A7C15ull ^ ((uint64_t)len * 0xC2B2AE3D27D4EB4Full);
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if (8 * i < len) h = hash_round(h, ch[i]);
    for (int64_t i = 32; i < len; i += 8) h = hash_round(h, chunk_at(c, pos + i, (int)(len - i < 8 ? len - i : 8)));
    return fmix64(h);
}

// 64-bit hash of the string at [pos, pos + len): a multiply-xorshift round
// per 8-byte chunk, seeded with the length, finished with fmix64.
__device__ __forceinline__ uint64_t str_hash(const char_span& c, int64_t pos, int64_t len) {
    uint64_t ch[4];
    load32(c, pos, len, ch);
    return str_hash_chunks(c, pos, len, ch);
}

// Does the string at [pa, pa + la) equal the one at pb whose first 32 bytes
// are in chb (load32)?
__device__ __forceinline__ bool str_eq_chunks(const char_span& c, int64_t pa, int64_t la, int64_t pb, int64_t lb,
                                              const uint64_t (&chb)[4]) {
    if (la != lb) return false;
    uint64_t cha[4];
    load32(c, pa, la, cha);
    bool eq = true;
#pragma unroll
    for (int i = 0; i < 4; ++i) eq &= cha[i] == chb[i];
    for (int64_t i = 32; eq && i < la; i += 8) {
        const int n = (int)(la - i < 8 ? la - i : 8);
        eq = chunk_at(c, pa + i, n) == chunk_at(c, pb + i, n);
    }
    return eq;
}

// Find or insert row r's string; returns the slot (or -1 on a full table).
//
// A new slot's inserter takes the next dictionary code, writes the string's
// first 32 bytes and length to the key store at that code, fences, and only
// then publishes the code in code_of_slot.  A row whose tag matches compares
// against the key store when the slot's code is published (one aligned
// 32-byte read), and against the slot's representative row in the input
// otherwise (or for the bytes past 32) — it never waits on an inserter.
// Without KEYSTORE (the plain engine's encoder, which numbers the slots
// itself) every compare reads the representative row.
template <bool KEYSTORE>
__device__ __forceinline__ int64_t find_or_insert(const batch_dev& b, const inst_dev& in, int inst_id, int64_t r,
                                                  int64_t o0, int64_t len, bool* inserted) {
    *inserted = false;
    const char_span sp{reinterpret_cast<const unsigned char*>(in.chars), in.clo, in.chi};
    uint64_t ch[4];
    load32(sp, o0, len, ch);
    const uint64_t h = str_hash_chunks(sp, o0, len, ch);
    const uint64_t tag = h >> 40;
    const uint64_t mine = (tag << 40) | (uint64_t)(r + 1);
    const uint32_t mask = b.slots - 1;
    uint32_t slot = (uint32_t)h & mask;
    unsigned long long* tab = b.entries + in.table_off;
    for (uint32_t p = 0; p <= mask; ++p) {
        unsigned long long e = ((volatile unsigned long long*)tab)[slot];
        const unsigned code = KEYSTORE ? ((const volatile unsigned*)b.code_of_slot)[in.table_off + slot] : ~0u;
        if (e == 0) {
            unsigned long long old = atomicCAS(tab + slot, 0ull, (unsigned long long)mine);
            if (old == 0) {
                *inserted = true;
                if (!KEYSTORE) return in.table_off + slot;
                const unsigned c = atomicAdd(&b.dict_size[inst_id], 1u);
                if (c < b.max_distinct) {
                    ulonglong2* k = reinterpret_cast<ulonglong2*>(b.ks_key + ((size_t)in.result_off + c) * 4);
                    k[0] = make_ulonglong2(ch[0], ch[1]);
                    k[1] = make_ulonglong2(ch[2], ch[3]);
                    b.ks_len[in.result_off + c] = (unsigned)len;
                    b.slot_of_code[in.result_off + c] = slot;
                    __threadfence();
                }
                ((volatile unsigned*)b.code_of_slot)[in.table_off + slot] = c;
                return in.table_off + slot;
            }
            e = old;
        }
        if ((e >> 40) == tag) {
            bool eq;
            if (code < b.max_distinct) {
                // Read at L2 (__ldcg): the key store is rewritten by every run
                // of the plan, and an SM's L1 may still hold an earlier run's
                // bytes at these addresses.
                const ulonglong2* k = reinterpret_cast<const ulonglong2*>(b.ks_key + ((size_t)in.result_off + code) * 4);
                const ulonglong2 k0 = __ldcg(k), k1 = __ldcg(k + 1);
                eq = __ldcg(b.ks_len + in.result_off + code) == (unsigned)len && k0.x == ch[0] && k0.y == ch[1] &&
                     k1.x == ch[2] && k1.y == ch[3];
                if (eq && len > 32) {
                    const int64_t rr = (int64_t)(e & ROW_MASK) - 1, pa = in.offsets[rr];
                    for (int64_t i = 32; eq && i < len; i += 8) {
                        const int nb = (int)(len - i < 8 ? len - i : 8);
                        eq = chunk_at(sp, pa + i, nb) == chunk_at(sp, o0 + i, nb);
                    }
                }
            } else {
                const int64_t rr = (int64_t)(e & ROW_MASK) - 1;
                eq = str_eq_chunks(sp, in.offsets[rr], in.offsets[rr + 1] - in.offsets[rr], o0, len, ch);
            }
            if (eq) return in.table_off + slot;
        }
        slot = (slot + 1) & mask;
    }
    atomicExch(b.overflow, 1);
    (void)inst_id;
    return -1;
}

// Four 256-thread blocks per SM (at most 64 registers): the kernel waits on
// dependent L2 accesses (offsets, string words, table entry, representative
// row), so resident warps matter more than registers.
__global__ void __launch_bounds__(256, 4) k_batch_main(batch_dev b) {
    __shared__ long long s_item;
    __shared__ inst_dev s_in;
    for (;;) {
        if (threadIdx.x == 0) {
            unsigned long long w = atomicAdd(b.work_counter, 1ull);
            s_item = w < (unsigned long long)b.n_work ? (long long)w : -1;
        }
        __syncthreads();
        const long long w = s_item;
        __syncthreads();
        if (w < 0) break;
        const work_item it = b.work[w];
        // The work item's instance stays in shared memory (read per use):
        // held in registers it cost every thread ~20 of them.
        if (threadIdx.x == 0) s_in = b.inst[it.inst];
        __syncthreads();
        const inst_dev& in = s_in;
        // A row's offsets, date and amount are loaded one iteration ahead,
        // so the dependent chain of a row starts at its string bytes.
        int64_t r = it.begin + threadIdx.x;
        int64_t o0 = 0, o1 = 0, am = 0;
        int32_t dt = 0;
        if (r < it.end) {
            o0 = in.offsets[r];
            o1 = in.offsets[r + 1];
            dt = in.date[r];
            am = in.amount[r];
        }
        for (; r < it.end; r += blockDim.x) {
            const int64_t rn = r + blockDim.x;
            int64_t n0 = 0, n1 = 0, nam = 0;
            int32_t ndt = 0;
            if (rn < it.end) {
                n0 = in.offsets[rn];
                n1 = in.offsets[rn + 1];
                ndt = in.date[rn];
                nam = in.amount[rn];
            }
            // The date range is applied before the string is encoded: the
            // output covers kept rows only, so a dropped row needs no hash,
            // probe or string bytes (its codes would never be read).
            if (dt >= in.lo && dt < in.hi) {
                bool ins;
                const int64_t slot = find_or_insert<true>(b, in, it.inst, r, o0, o1 - o0, &ins);
                if (slot >= 0) {
                    atomicAdd(&b.sum_slot[slot], (unsigned long long)am);
                    atomicAdd(&b.cnt_slot[slot], 1ull);
                }
            }
            o0 = n0;
            o1 = n1;
            dt = ndt;
            am = nam;
        }
    }
}

// Per-code results (grid over all instances' codes): each code's slot gives
// its first row, SUM and COUNT.  The finalize also returns the slots it read
// to their empty state, so the next run of the plan starts from clean tables
// without clearing every slot (after an overflow the host clears them all).
// Lanes of a warp that share an instance add their kept groups with one
// atomic.
__global__ void k_batch_finalize(batch_dev b, int n_inst) {
    const int64_t total = (int64_t)n_inst * b.max_distinct;
    const int lane = threadIdx.x & 31;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < total; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = base + threadIdx.x;
        int inst = -1;
        bool kept = false;
        if (o < total) {
            inst = (int)(o / b.max_distinct);
            const uint32_t code = (uint32_t)(o - (int64_t)inst * b.max_distinct);
            const unsigned nd = b.dict_size[inst];
            if (nd > b.max_distinct && code == 0) atomicExch(b.overflow, 1);
            if (code < nd) {
                const int64_t g = b.inst[inst].table_off + b.slot_of_code[o];
                const unsigned long long c = b.cnt_slot[g];
                b.out_sum[o] = (long long)b.sum_slot[g];
                b.out_cnt[o] = (long long)c;
                b.out_first[o] = (long long)(b.entries[g] & ROW_MASK) - 1;
                kept = c != 0;
                b.entries[g] = 0;
                b.sum_slot[g] = 0;
                b.cnt_slot[g] = 0;
                b.code_of_slot[g] = ~0u;
            }
        }
        const unsigned same = __match_any_sync(0xffffffffu, inst);
        const unsigned hits = __ballot_sync(0xffffffffu, kept) & same;
        if (inst >= 0 && hits && lane == __ffs(same) - 1)
            atomicAdd((unsigned long long*)&b.out_groups[inst], (unsigned long long)__popc(hits));
    }
}

// ---- plain-engine pieces -------------------------------------------------
struct enc_dev {
    const char* chars;
    const int64_t* offsets;
    int64_t rows;
    unsigned long long* entries;
    unsigned* code_of_slot;
    unsigned* dict_size;
    int* overflow;
    uint32_t slots;
    int32_t* codes;
    int64_t clo, chi;  // byte range of chars the strings occupy: offsets[0], offsets[rows]
};

__device__ __forceinline__ int64_t enc_find(const enc_dev& e, int64_t r, bool insert, bool* inserted) {
    batch_dev b;
    b.entries = e.entries;
    b.slots = e.slots;
    b.overflow = e.overflow;
    inst_dev in;
    in.chars = e.chars;
    in.offsets = e.offsets;
    in.table_off = 0;
    in.clo = e.clo;
    in.chi = e.chi;
    if (insert) return find_or_insert<false>(b, in, 0, r, e.offsets[r], e.offsets[r + 1] - e.offsets[r], inserted);
    // lookup only: the insert pass has published every string
    *inserted = false;
    const char_span sp{reinterpret_cast<const unsigned char*>(e.chars), e.clo, e.chi};
    const int64_t o0 = e.offsets[r], len = e.offsets[r + 1] - o0;
    uint64_t ch[4];
    load32(sp, o0, len, ch);
    const uint64_t h = str_hash_chunks(sp, o0, len, ch), tag = h >> 40;
    const uint32_t mask = e.slots - 1;
    uint32_t slot = (uint32_t)h & mask;
    for (uint32_t p = 0; p <= mask; ++p) {
        unsigned long long en = e.entries[slot];
        if (en == 0) return -1;
        if ((en >> 40) == tag) {
            int64_t rr = (int64_t)(en & ROW_MASK) - 1;
            if (str_eq_chunks(sp, e.offsets[rr], e.offsets[rr + 1] - e.offsets[rr], o0, len, ch)) return slot;
        }
        slot = (slot + 1) & mask;
    }
    return -1;
}

__global__ void k_enc_insert(enc_dev e) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < e.rows; r += (int64_t)gridDim.x * blockDim.x) {
        bool ins;
        int64_t s = enc_find(e, r, true, &ins);
        if (s >= 0 && ins) e.code_of_slot[s] = atomicAdd(e.dict_size, 1u);
    }
}
__global__ void k_enc_lookup(enc_dev e) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < e.rows; r += (int64_t)gridDim.x * blockDim.x) {
        bool ins;
        int64_t s = enc_find(e, r, false, &ins);
        e.codes[r] = s >= 0 ? (int32_t)e.code_of_slot[s] : -1;
    }
}

// Filter with compaction: rows with lo <= date < hi keep (code, amount).
constexpr int FT = 256, FIPT = 8;
__global__ void __launch_bounds__(FT) k_filter_count(const int32_t* __restrict__ date, int64_t n, int32_t lo, int32_t hi,
                                                     int64_t* __restrict__ tile_cnt) {
    int64_t base = blockIdx.x * (int64_t)FT * FIPT;
    int c = 0;
    for (int k = 0; k < FIPT; ++k) {
        int64_t i = base + k * FT + threadIdx.x;
        if (i < n) c += date[i] >= lo && date[i] < hi;
    }
    __shared__ int sm[FT / 32];
    int w = dev_::warp_sum(c);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int j = 0; j < FT / 32; ++j) t += sm[j];
        tile_cnt[blockIdx.x] = t;
    }
}
__global__ void __launch_bounds__(FT) k_filter_write(const int32_t* __restrict__ date, const int32_t* __restrict__ codes,
                                                     const int64_t* __restrict__ amount, int64_t n, int32_t lo,
                                                     int32_t hi, const int64_t* __restrict__ tile_off,
                                                     int32_t* __restrict__ out_codes, int64_t* __restrict__ out_amt) {
    __shared__ int64_t sm[FT / 32 + 1];
    int64_t base = blockIdx.x * (int64_t)FT * FIPT;
    int64_t run = tile_off[blockIdx.x];
    for (int k = 0; k < FIPT; ++k) {
        int64_t i = base + k * FT + threadIdx.x;
        int keep = (i < n && date[i] >= lo && date[i] < hi) ? 1 : 0;
        int64_t total;
        int64_t pos = run + dev_::block_exclusive_sum<FT, int64_t>(keep, sm, &total);
        if (keep) {
            out_codes[pos] = codes[i];
            out_amt[pos] = amount[i];
        }
        run += total;
    }
}

__global__ void k_scatter_codes(const int32_t* __restrict__ gcode, const int64_t* __restrict__ gsum,
                                const int64_t* __restrict__ gcnt, int64_t groups, long long* __restrict__ out_sum,
                                long long* __restrict__ out_cnt) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < groups; g += (int64_t)gridDim.x * blockDim.x) {
        out_sum[gcode[g]] = gsum[g];
        out_cnt[gcode[g]] = gcnt[g];
    }
}
__global__ void k_first_rows(const unsigned long long* __restrict__ entries, const unsigned* __restrict__ code_of_slot,
                             uint32_t slots, long long* __restrict__ out_first) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < slots; s += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long e = entries[s];
        if (e) out_first[code_of_slot[s]] = (long long)(e & ROW_MASK) - 1;
    }
}

}  // namespace
}  // namespace gx

struct gx_batch_plan {
    std::vector<gx_batch_instance> inst;
    std::vector<int64_t> span_lo, span_hi;  // per instance: offsets[0], offsets[rows]
    std::vector<gx::inst_dev> hinst;
    int64_t max_distinct = 0;
    uint32_t slots = 0;
    int tile_rows = 4096;
    int lf_pct = 50;
    gx::dbuf d_inst, d_work, entries, code_of_slot, sum_slot, cnt_slot, dict_size, ctrl, ks_key, ks_len, slot_of_code;
    gx::dbuf out_sum, out_cnt, out_first, out_groups;
    int64_t n_work = 0;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t capture_stream = nullptr;  // private: the legacy default stream cannot be captured
    bool last_plain = false;
    ~gx_batch_plan() {
        if (graph) cudaGraphExecDestroy(graph);
        if (capture_stream) cudaStreamDestroy(capture_stream);
    }
};

namespace gx {

// Every slot empty: entry 0, no code, zero SUM and COUNT.
static void clear_tables(gx_batch_plan* p, cudaStream_t s) {
    const size_t total_slots = p->inst.size() * (size_t)p->slots;
    GX_CUDA(cudaMemsetAsync(p->entries.get(), 0, total_slots * 8, s));
    GX_CUDA(cudaMemsetAsync(p->code_of_slot.get(), 0xFF, total_slots * 4, s));
    GX_CUDA(cudaMemsetAsync(p->sum_slot.get(), 0, total_slots * 8, s));
    GX_CUDA(cudaMemsetAsync(p->cnt_slot.get(), 0, total_slots * 8, s));
}

static void batch_layout(gx_batch_plan* p, int tile, int lf, cudaStream_t s) {
    const int n = (int)p->inst.size();
    p->tile_rows = tile;
    p->lf_pct = lf;
    p->slots = (uint32_t)next_pow2((uint64_t)std::max<int64_t>(64, p->max_distinct * 100 / lf + 1));
    std::vector<work_item> work;
    p->hinst.resize(n);
    for (int i = 0; i < n; ++i) {
        const gx_batch_instance& b = p->inst[i];
        inst_dev d;
        d.chars = b.chars;
        d.offsets = b.offsets;
        d.date = b.date;
        d.amount = b.amount;
        d.rows = b.rows;
        d.lo = b.date_lo;
        d.hi = b.date_hi;
        d.table_off = (int64_t)i * p->slots;
        d.result_off = (int64_t)i * p->max_distinct;
        d.clo = p->span_lo[i];
        d.chi = p->span_hi[i];
        p->hinst[i] = d;
        for (int64_t r = 0; r < b.rows; r += tile) work.push_back({i, 0, r, std::min<int64_t>(b.rows, r + tile)});
    }
    p->n_work = (int64_t)work.size();
    p->d_inst = dbuf(sizeof(inst_dev) * std::max(n, 1), s);
    p->d_work = dbuf(sizeof(work_item) * std::max<int64_t>(p->n_work, 1), s);
    GX_CUDA(cudaMemcpyAsync(p->d_inst.get(), p->hinst.data(), sizeof(inst_dev) * n, cudaMemcpyHostToDevice, s));
    if (p->n_work)
        GX_CUDA(cudaMemcpyAsync(p->d_work.get(), work.data(), sizeof(work_item) * p->n_work, cudaMemcpyHostToDevice, s));
    const size_t total_slots = (size_t)n * p->slots;
    p->entries = dbuf(total_slots * 8, s);
    p->code_of_slot = dbuf(total_slots * 4, s);
    p->sum_slot = dbuf(total_slots * 8, s);
    p->cnt_slot = dbuf(total_slots * 8, s);
    p->dict_size = dbuf((size_t)std::max(n, 1) * 4, s);
    p->ctrl = dbuf(16, s);
    const size_t total_codes = (size_t)n * p->max_distinct;
    p->out_sum = dbuf(std::max<size_t>(total_codes, 1) * 8, s);
    p->out_cnt = dbuf(std::max<size_t>(total_codes, 1) * 8, s);
    p->out_first = dbuf(std::max<size_t>(total_codes, 1) * 8, s);
    p->out_groups = dbuf((size_t)std::max(n, 1) * 8, s);
    p->ks_key = dbuf(std::max<size_t>(total_codes, 1) * 32, s);
    p->ks_len = dbuf(std::max<size_t>(total_codes, 1) * 4, s);
    p->slot_of_code = dbuf(std::max<size_t>(total_codes, 1) * 4, s);
    clear_tables(p, s);
    GX_CUDA(cudaStreamSynchronize(s));
    if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
}

static batch_dev batch_view(gx_batch_plan* p) {
    batch_dev b;
    b.inst = p->d_inst.get<inst_dev>();
    b.work = p->d_work.get<work_item>();
    b.n_work = p->n_work;
    b.entries = p->entries.get<unsigned long long>();
    b.code_of_slot = p->code_of_slot.get<unsigned>();
    b.sum_slot = p->sum_slot.get<unsigned long long>();
    b.cnt_slot = p->cnt_slot.get<unsigned long long>();
    b.dict_size = p->dict_size.get<unsigned>();
    b.ks_key = p->ks_key.get<unsigned long long>();
    b.ks_len = p->ks_len.get<unsigned>();
    b.slot_of_code = p->slot_of_code.get<unsigned>();
    b.work_counter = p->ctrl.get<unsigned long long>();
    b.overflow = reinterpret_cast<int*>(p->ctrl.get<char>() + 8);
    b.slots = p->slots;
    b.max_distinct = (uint32_t)p->max_distinct;
    b.out_sum = p->out_sum.get<long long>();
    b.out_cnt = p->out_cnt.get<long long>();
    b.out_first = p->out_first.get<long long>();
    b.out_groups = p->out_groups.get<long long>();
    return b;
}

// The whole batched run as stream work (resets, main, finalize).
static void batch_enqueue(gx_batch_plan* p, cudaStream_t s, bool count_launches = true) {
    const int n = (int)p->inst.size();
    const size_t total_codes = (size_t)n * p->max_distinct;
    // The slot tables are clean here: set up once by batch_layout and
    // returned to empty by the previous run's finalize.
    GX_CUDA(cudaMemsetAsync(p->dict_size.get(), 0, (size_t)n * 4, s));
    GX_CUDA(cudaMemsetAsync(p->ctrl.get(), 0, 16, s));
    GX_CUDA(cudaMemsetAsync(p->out_sum.get(), 0, total_codes * 8, s));
    GX_CUDA(cudaMemsetAsync(p->out_cnt.get(), 0, total_codes * 8, s));
    GX_CUDA(cudaMemsetAsync(p->out_first.get(), 0xFF, total_codes * 8, s));
    GX_CUDA(cudaMemsetAsync(p->out_groups.get(), 0, (size_t)n * 8, s));
    batch_dev b = batch_view(p);
    k_batch_main<<<dev().sm_count * 8, 256, 0, s>>>(b);
    GX_CUDA(cudaGetLastError());
    k_batch_finalize<<<grid_for((int64_t)std::max<size_t>(total_codes, 1), 256, 8), 256, 0, s>>>(b, n);
    GX_CUDA(cudaGetLastError());
    if (count_launches) g_launches.fetch_add(2);
}

static float time_batch(gx_batch_plan* p, cudaStream_t s) {
    cudaEvent_t a, b;
    GX_CUDA(cudaEventCreate(&a));
    GX_CUDA(cudaEventCreate(&b));
    batch_enqueue(p, s);  // warm
    GX_CUDA(cudaEventRecord(a, s));
    batch_enqueue(p, s);
    GX_CUDA(cudaEventRecord(b, s));
    GX_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

// Autotuner: time each (tile rows, load factor) candidate on this batch.
static void batch_autotune(gx_batch_plan* p, cudaStream_t s) {
    const int tiles[] = {1024, 4096, 16384};
    const int lfs[] = {25, 50};
    float best = 1e30f;
    int bt = 4096, bl = 50;
    if (const char* e = getenv("GX_BATCH_TILE")) {
        batch_layout(p, atoi(e), 50, s);
        return;
    }
    for (int t : tiles)
        for (int l : lfs) {
            batch_layout(p, t, l, s);
            float ms = time_batch(p, s);
            if (ms < best) { best = ms; bt = t; bl = l; }
        }
    batch_layout(p, bt, bl, s);
}

static void check_overflow(gx_batch_plan* p, cudaStream_t s) {
    int ovf = read_scalar(reinterpret_cast<int*>(p->ctrl.get<char>() + 8), s);
    if (ovf) {
        // Slots past max_distinct were never listed for the finalize to clear.
        clear_tables(p, s);
        GX_CUDA(cudaStreamSynchronize(s));
        fail(GX_EOVERFLOW, "batch: an instance exceeded max_distinct or its table filled");
    }
}

static void batch_run(gx_batch_plan* p, cudaStream_t s) {
    if (!p->graph) {
        // Capture once on the plan's own stream; the executable graph is then
        // launched on whatever stream the caller passes.
        if (!p->capture_stream) GX_CUDA(cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking));
        GX_CUDA(cudaStreamSynchronize(s));  // the capture records work only; inputs are ready
        cudaGraph_t g = nullptr;
        GX_CUDA(cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeThreadLocal));
        try {
            batch_enqueue(p, p->capture_stream, false);
        } catch (...) {
            cudaStreamEndCapture(p->capture_stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        GX_CUDA(cudaStreamEndCapture(p->capture_stream, &g));
        cudaError_t e = cudaGraphInstantiate(&p->graph, g, 0);
        cudaGraphDestroy(g);
        GX_CUDA(e);
    }
    GX_CUDA(cudaGraphLaunch(p->graph, s));
    g_launches.fetch_add(2);
    check_overflow(p, s);
    p->last_plain = false;
}

// The same pipeline as one operator sequence per instance.
static void batch_run_plain(gx_batch_plan* p, cudaStream_t s) {
    const int n = (int)p->inst.size();
    const size_t total_codes = (size_t)n * p->max_distinct;
    GX_CUDA(cudaMemsetAsync(p->out_sum.get(), 0, total_codes * 8, s));
    GX_CUDA(cudaMemsetAsync(p->out_cnt.get(), 0, total_codes * 8, s));
    GX_CUDA(cudaMemsetAsync(p->out_first.get(), 0xFF, total_codes * 8, s));
    std::vector<long long> groups(n, 0);
    for (int i = 0; i < n; ++i) {
        const gx_batch_instance& b = p->inst[i];
        const int64_t rows = b.rows;
        // 1. string dictionary encode
        uint32_t slots = (uint32_t)next_pow2((uint64_t)std::max<int64_t>(64, p->max_distinct * 2));
        dbuf ent((size_t)slots * 8, s), cos((size_t)slots * 4, s), ds(16, s), codes((size_t)std::max<int64_t>(rows, 1) * 4, s);
        GX_CUDA(cudaMemsetAsync(ent.get(), 0, (size_t)slots * 8, s));
        GX_CUDA(cudaMemsetAsync(ds.get(), 0, 16, s));
        enc_dev e{b.chars, b.offsets, rows, ent.get<unsigned long long>(), cos.get<unsigned>(), ds.get<unsigned>(),
                  reinterpret_cast<int*>(ds.get<char>() + 8), slots, codes.get<int32_t>(), p->span_lo[i],
                  p->span_hi[i]};
        if (rows > 0) {
            k_enc_insert<<<grid_for(rows, 256, 4), 256, 0, s>>>(e);
            GX_LAUNCHED();
            k_enc_lookup<<<grid_for(rows, 256, 4), 256, 0, s>>>(e);
            GX_LAUNCHED();
        }
        unsigned hds[4];
        GX_CUDA(cudaMemcpyAsync(hds, ds.get(), 16, cudaMemcpyDeviceToHost, s));
        GX_CUDA(cudaStreamSynchronize(s));
        if (hds[2] || hds[0] > (unsigned)p->max_distinct) fail(GX_EOVERFLOW, "batch: max_distinct exceeded");
        // 2. filter with compaction
        int64_t ntiles = ceil_div(std::max<int64_t>(rows, 1), FT * FIPT);
        dbuf tc(ntiles * 8, s), toff((ntiles + 1) * 8, s);
        k_filter_count<<<(unsigned)ntiles, FT, 0, s>>>(b.date, rows, b.date_lo, b.date_hi, tc.get<int64_t>());
        GX_LAUNCHED();
        exclusive_scan_i64(tc.get<int64_t>(), toff.get<int64_t>(), ntiles, s);
        int64_t kept = read_scalar(toff.get<int64_t>() + ntiles, s);
        dbuf kc((size_t)std::max<int64_t>(kept, 1) * 4, s), ka((size_t)std::max<int64_t>(kept, 1) * 8, s);
        k_filter_write<<<(unsigned)ntiles, FT, 0, s>>>(b.date, codes.get<int32_t>(), b.amount, rows, b.date_lo,
                                                      b.date_hi, toff.get<int64_t>(), kc.get<int32_t>(),
                                                      ka.get<int64_t>());
        GX_LAUNCHED();
        // 3. hash group-by on the codes: SUM(amount), COUNT
        gx_column_view vv{ka.get(), kept, GX_INT64, 0};
        gx_table_view vt{&vv, 1};
        gx_agg_request req[2] = {{0, GX_AGG_SUM}, {0, GX_AGG_COUNT_ALL}};
        agg_plan plan = make_agg_plan(&vt, req, 2, false);
        gx_groupby_hint hint;
        gx_groupby_hint_init(&hint);
        hint.groups_upper_bound = std::max<int64_t>(1, hds[0]);
        hint.groupby_algo = GX_GB_HASH;
        col kcol;
        kcol.data = kc.get();
        kcol.n = kept;
        kcol.type = GX_INT32;
        gx_table t;
        hash_groupby(kcol, plan, &hint, s, &t);
        const int64_t ng = t.cols[0].size;
        const int64_t off = (int64_t)i * p->max_distinct;
        if (ng > 0) {
            k_scatter_codes<<<grid_for(ng, 256, 4), 256, 0, s>>>(t.cols[0].buf.get<int32_t>(), t.cols[1].buf.get<int64_t>(),
                                                                t.cols[2].buf.get<int64_t>(), ng, p->out_sum.get<long long>() + off,
                                                                p->out_cnt.get<long long>() + off);
            GX_LAUNCHED();
        }
        k_first_rows<<<grid_for(slots, 256, 4), 256, 0, s>>>(ent.get<unsigned long long>(), cos.get<unsigned>(), slots,
                                                           p->out_first.get<long long>() + off);
        GX_LAUNCHED();
        groups[i] = ng;
        GX_CUDA(cudaStreamSynchronize(s));
    }
    GX_CUDA(cudaMemcpyAsync(p->out_groups.get(), groups.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
    GX_CUDA(cudaStreamSynchronize(s));
    p->last_plain = true;
}

// Hash dictionary encode of one ARROW string column: int32 codes, dense in
// [0, NDV) in first-insert order (the reference's hash encode semantics for
// numeric keys, src/cuda/compress/dictionary_encode.cu:71-96; its
// dictionary_encode rejects STRING, dictionary_encode.cu:32-34).  The table
// is the plain engine's (hash tag + representative row per slot); without a
// size hint it starts at 2^22 distinct strings and grows by 4x on overflow.
void dictionary_encode_strings(const gx_column_view& v, int64_t size_hint, cudaStream_t s, gx_column* out,
                               int64_t* ndv) {
    require(v.type == GX_STRING, "dictionary_encode_strings: STRING column required");
    require(v.size >= 0 && v.offset >= 0, "dictionary_encode_strings: negative size or offset");
    const int64_t rows = v.size;
    owned_col codes = make_col(GX_INT32, rows, s);
    int64_t distinct = 0;
    if (rows > 0) {
        require(v.data != nullptr, "dictionary_encode_strings: null string columns");
        const gx_string_columns* sc = static_cast<const gx_string_columns*>(v.data);
        require(sc->chars && sc->offsets, "dictionary_encode_strings: null chars or offsets");
        int64_t bound = size_hint > 0 ? std::min(size_hint, rows) : std::min<int64_t>(rows, 1 << 22);
        // Byte range of chars these rows' strings occupy (reads stay inside it).
        int64_t span[2];
        GX_CUDA(cudaMemcpyAsync(&span[0], sc->offsets + v.offset, 8, cudaMemcpyDeviceToHost, s));
        GX_CUDA(cudaMemcpyAsync(&span[1], sc->offsets + v.offset + rows, 8, cudaMemcpyDeviceToHost, s));
        GX_CUDA(cudaStreamSynchronize(s));
        bool done = false;
        for (int attempt = 0; attempt < 8 && !done; ++attempt) {
            uint32_t slots = (uint32_t)next_pow2((uint64_t)std::max<int64_t>(64, 2 * bound));
            dbuf ent((size_t)slots * 8, s), cos((size_t)slots * 4, s), ds(16, s);
            GX_CUDA(cudaMemsetAsync(ent.get(), 0, (size_t)slots * 8, s));
            GX_CUDA(cudaMemsetAsync(ds.get(), 0, 16, s));
            enc_dev e{sc->chars, sc->offsets + v.offset, rows, ent.get<unsigned long long>(), cos.get<unsigned>(),
                      ds.get<unsigned>(), reinterpret_cast<int*>(ds.get<char>() + 8), slots, codes.buf.get<int32_t>(),
                      span[0], span[1]};
            k_enc_insert<<<grid_for(rows, 256, 4), 256, 0, s>>>(e);
            GX_LAUNCHED();
            unsigned hds[4];
            GX_CUDA(cudaMemcpyAsync(hds, ds.get(), 16, cudaMemcpyDeviceToHost, s));
            GX_CUDA(cudaStreamSynchronize(s));
            if (hds[2]) {  // table full: grow
                require(bound < rows, "dictionary_encode_strings: table overflow");
                bound = std::min(rows, bound * 4);
                continue;
            }
            k_enc_lookup<<<grid_for(rows, 256, 4), 256, 0, s>>>(e);
            GX_LAUNCHED();
            GX_CUDA(cudaStreamSynchronize(s));
            distinct = hds[0];
            done = true;
        }
        require(done, "dictionary_encode_strings: table overflow after retries");
    }
    *ndv = distinct;
    *out = to_gx_column(std::move(codes));
}

}  // namespace gx

#define GX_BTRY(...)                                       \
    try {                                                  \
        __VA_ARGS__;                                       \
        return GX_OK;                                      \
    } catch (const gx::error& e) {                         \
        gx::set_last_error(e.what());                      \
        return e.status;                                   \
    } catch (const std::exception& e) {                    \
        gx::set_last_error(e.what());                      \
        return GX_EINVAL;                                  \
    }

namespace gx {
void set_last_error(const char* msg);
}

extern "C" {

gx_status gx_batch_plan_create(const gx_batch_instance* instances, int32_t count, int64_t max_distinct, gx_stream_t st,
                               gx_batch_plan** plan) {
    GX_BTRY({
        gx::require(plan != nullptr && (count == 0 || instances != nullptr), "batch: bad arguments");
        gx::require(count > 0, "batch: no instances");
        gx::require(max_distinct > 0 && max_distinct < (1ll << 30), "batch: max_distinct out of range");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(st);
        std::unique_ptr<gx_batch_plan> p(new gx_batch_plan);
        for (int i = 0; i < count; ++i) {
            const gx_batch_instance& b = instances[i];
            gx::require(b.rows >= 0 && b.rows < (1ll << 39), "batch: instance row count out of range");
            gx::require(b.rows == 0 || (b.chars && b.offsets && b.date && b.amount), "batch: null column pointer");
            p->inst.push_back(b);
        }
        // Byte range of chars each instance's strings occupy: offsets[0] and
        // offsets[rows], read once (string reads stay inside it).
        p->span_lo.assign(count, 0);
        p->span_hi.assign(count, 0);
        for (int i = 0; i < count; ++i)
            if (instances[i].rows > 0) {
                GX_CUDA(cudaMemcpyAsync(&p->span_lo[i], instances[i].offsets, 8, cudaMemcpyDeviceToHost, s));
                GX_CUDA(cudaMemcpyAsync(&p->span_hi[i], instances[i].offsets + instances[i].rows, 8,
                                        cudaMemcpyDeviceToHost, s));
            }
        GX_CUDA(cudaStreamSynchronize(s));
        p->max_distinct = max_distinct;
        gx::batch_autotune(p.get(), s);
        *plan = p.release();
    })
}
gx_status gx_batch_run(gx_batch_plan* plan, gx_stream_t st) {
    GX_BTRY({
        gx::require(plan != nullptr, "batch: null plan");
        gx::batch_run(plan, reinterpret_cast<cudaStream_t>(st));
    })
}
gx_status gx_batch_run_per_instance(gx_batch_plan* plan, gx_stream_t st) {
    GX_BTRY({
        gx::require(plan != nullptr, "batch: null plan");
        gx::batch_run_plain(plan, reinterpret_cast<cudaStream_t>(st));
    })
}
gx_status gx_batch_results(const gx_batch_plan* plan, gx_batch_result* res) {
    GX_BTRY({
        gx::require(plan && res, "batch: null argument");
        const int n = (int)plan->inst.size();
        std::vector<long long> groups(n);
        GX_CUDA(cudaMemcpy(groups.data(), plan->out_groups.get(), (size_t)n * 8, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i) {
            const int64_t off = (int64_t)i * plan->max_distinct;
            res[i].num_groups = groups[i];
            res[i].sum = plan->out_sum.get<int64_t>() + off;
            res[i].count = plan->out_cnt.get<int64_t>() + off;
            res[i].first_row = plan->out_first.get<int64_t>() + off;
        }
    })
}
gx_status gx_batch_tuning(const gx_batch_plan* plan, int32_t* tile_rows, int32_t* lf) {
    GX_BTRY({
        gx::require(plan && tile_rows && lf, "batch: null argument");
        *tile_rows = plan->tile_rows;
        *lf = plan->lf_pct;
    })
}
void gx_batch_plan_free(gx_batch_plan* plan) {
    delete plan;  // the destructor releases the graph and the capture stream
}

gx_status gx_dictionary_encode_strings(gx_column_view col, int64_t dictionary_size_hint, gx_stream_t st,
                                       gx_column* codes, int64_t* dict_size) {
    GX_BTRY({
        gx::require(codes && dict_size, "null output");
        gx::dictionary_encode_strings(col, dictionary_size_hint, reinterpret_cast<cudaStream_t>(st), codes,
                                      dict_size);
    })
}

}  // extern "C"
