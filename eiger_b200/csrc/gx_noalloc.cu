// gx_noalloc.cu — gx_sort_column_pair_noalloc: the stable (key, value) radix
// sort of gx_sort_column_pair, writing into caller buffers and allocating
// nothing.
//
// Who needs it: a host engine that hands all of HBM to its own buffer
// manager before any operator runs leaves no room for the library's pool, and
// an engine that keeps a latency budget per operator cannot afford the device
// synchronisation that cudaMalloc / cudaFree (or growing a memory pool) may
// imply.  Both still want a sort.  This entry point takes every temporary —
// ping-pong halves, per-tile digit counts and offsets, the scan's levels —
// from one fixed array in device memory declared below, and returns its
// results in buffers the caller already owns.
//
// Limits and rules:
//   * scratch is NOALLOC_SCRATCH_BYTES (8 MiB); a call whose sort needs more
//     (about 0.5 M pairs of 8+8 bytes, 1 M pairs of 4+4 bytes) fails with
//     GX_EINVAL before anything is launched;
//   * keys and values must be 4 or 8 bytes wide (1- and 2-byte columns need
//     widened copies, which the allocating entry point makes);
//   * nothing in the scratch has to start at zero: every byte a launch reads
//     was written earlier in the same call;
//   * all calls on one device share the one array, so two calls whose work
//     overlaps on the device (different streams with no ordering between
//     them, or concurrent host threads on different streams) race and corrupt
//     each other's results; order them on one stream or with events;
//   * the first call on each device resolves the array's device address with
//     cudaGetSymbolAddress (which may load this file's device code) and raises
//     the shared-memory limit of the scatter kernel for all four 4/8-byte
//     (key, value) width pairs, whatever widths that call sorts; make that
//     first call before any stream capture begins.  Later calls, of any width
//     pair, only launch kernels and queue device-to-device copies on
//     `stream`, and return without waiting.
#include <atomic>

#include "gx_groupby.h"

namespace gx {
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per device ordinal (dev() rejects
// ordinals of GX_MAX_DEVICES and above); null until that device's set-up ran.
std::atomic<void*> g_scratch_addr[GX_MAX_DEVICES];

char* noalloc_scratch() {
    const int d = dev().device;
    void* p = g_scratch_addr[d].load(std::memory_order_acquire);
    if (p == nullptr) {
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            (void)cudaGetLastError();
            fail(GX_ECUDA, std::string("sort_column_pair_noalloc: cudaGetSymbolAddress failed: ") +
                               cudaGetErrorString(e));
        }
        // Every width pair's scatter attribute now, so no later call changes one.
        radix_prepare_pair_scatters();
        g_scratch_addr[d].store(p, std::memory_order_release);
    }
    return static_cast<char*>(p);
}

bool fixed_width(int type) {
    int w = size_of(type);
    return is_numeric(type) && (w == 4 || w == 8);
}

bool overlaps(const void* a, size_t an, const void* b, size_t bn) {
    auto x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return an && bn && x < y + bn && y < x + an;
}

void sort_pair_noalloc(const gx_column_view& key, const gx_column_view& val, int begin_bit, int end_bit, int order,
                       void* key_out, void* val_out, cudaStream_t s) {
    if (key.size < 0 || key.offset < 0 || val.size < 0 || val.offset < 0)
        fail(GX_EINVAL, "sort_column_pair_noalloc: negative size or offset");
    if (key.size != val.size) fail(GX_EINVAL, "sort_column_pair_noalloc: key and value columns differ in length");
    if (!fixed_width(key.type) || !fixed_width(val.type))
        fail(GX_EUNSUPPORTED, "sort_column_pair_noalloc: keys and values must be 4- or 8-byte numeric columns");
    if (order != GX_ASCENDING && order != GX_DESCENDING) fail(GX_EINVAL, "sort_column_pair_noalloc: bad order");
    const int64_t n = key.size;
    const int kw = size_of(key.type), vw = size_of(val.type);
    const size_t need = radix_pairs_scratch_bytes(n, kw, vw);
    if (need > NOALLOC_SCRATCH_BYTES)
        fail(GX_EINVAL, "sort_column_pair_noalloc: " + std::to_string(n) + " pairs of " + std::to_string(kw) + "+" +
                            std::to_string(vw) + " bytes need " + std::to_string(need) +
                            " bytes of scratch, above the fixed limit of " + std::to_string(NOALLOC_SCRATCH_BYTES) +
                            " bytes (8 MiB); use gx_sort_column_pair");
    if (n == 0) return;
    if (!key.data || !val.data || !key_out || !val_out) fail(GX_EINVAL, "sort_column_pair_noalloc: null buffer");
    col k{static_cast<const char*>(key.data) + key.offset * kw, n, key.type};
    const void* v = static_cast<const char*>(val.data) + val.offset * vw;
    const size_t kb = (size_t)n * kw, vb = (size_t)n * vw;
    if (overlaps(key_out, kb, val_out, vb) || overlaps(key_out, kb, k.data, kb) || overlaps(key_out, kb, v, vb) ||
        overlaps(val_out, vb, k.data, kb) || overlaps(val_out, vb, v, vb))
        fail(GX_EINVAL, "sort_column_pair_noalloc: output buffers overlap each other or the inputs");
    radix_sort_pairs_scratch(k, v, vw, begin_bit, end_bit, order == GX_DESCENDING, key_out, val_out,
                             noalloc_scratch(), s);
}

}  // namespace
}  // namespace gx

extern "C" gx_status gx_sort_column_pair_noalloc(gx_column_view key, gx_column_view val, int32_t begin_bit,
                                                 int32_t end_bit, int32_t order, void* key_out, void* val_out,
                                                 gx_stream_t stream) {
    try {
        gx::sort_pair_noalloc(key, val, begin_bit, end_bit, order, key_out, val_out,
                              reinterpret_cast<cudaStream_t>(stream));
        gx::set_last_error("");
        return GX_OK;
    } catch (const gx::error& e) {
        gx::set_last_error(e.what());
        return e.status;
    } catch (const std::exception& e) {
        gx::set_last_error(e.what());
        return GX_EINVAL;
    }
}
