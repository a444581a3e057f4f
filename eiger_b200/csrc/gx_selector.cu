// gx_selector.cu — learned strategy selector for the group-by variants.
//
// The reference's AUTO rule is a fixed threshold on a full-column
// HyperLogLog estimate (src/cuda/operators/groupby/groupby.cu:68-119); this
// library keeps that rule as the fallback and as the baseline the selector's
// regret is compared with.  The selector instead sketches a 2^14-row strided
// sample (HyperLogLog estimate, exact sample distinct count, singleton
// fraction, top-8 key frequencies, a GEE extrapolation of the distinct count
// — Charikar, Chaudhuri, Motwani, Narasayya, PODS 2000) and scores the
// HASH / SORT / PARTITION variants and four partition fan-outs with a
// 3-layer MLP (20 -> 64 -> 64 -> 7, ReLU) whose weights are stored in FP16
// and whose arithmetic accumulates in FP32; 4 of its 20 inputs describe the
// aggregation list.  Training runs on the GPU with the forward / backward /
// Adam kernels below.
#include <algorithm>
#include <cmath>
#include <cuda_fp16.h>
#include <functional>
#include <mutex>

#include "gx_groupby.h"

namespace gx {

void hll_registers(const col& key_in, int64_t n, int64_t stride, unsigned* d_regs, cudaStream_t s);
double hll_estimate(const unsigned* regs);

constexpr int F = GX_SEL_NUM_FEATURES;
constexpr int H = GX_SEL_HIDDEN;
constexpr int O = GX_SEL_NUM_OUTPUTS;
constexpr int P_W1 = 0, P_B1 = P_W1 + H * F, P_W2 = P_B1 + H, P_B2 = P_W2 + H * H, P_W3 = P_B2 + H,
              P_B3 = P_W3 + O * H, P_TOTAL = P_B3 + O;
static const int FANOUT_BITS[GX_SEL_NUM_FANOUTS] = {8, 10, 12, 14};

namespace {

__global__ void k_sample(const void* __restrict__ keys, int width, int kind, int64_t m, int64_t stride,
                         unsigned long long* __restrict__ out) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = j * stride;
        uint64_t b;
        switch (width) {
            case 8: b = canon64(static_cast<const unsigned long long*>(keys)[i], kind); break;
            case 4: b = canon32(static_cast<const unsigned*>(keys)[i], kind); break;
            case 2: b = static_cast<const uint16_t*>(keys)[i]; break;
            default: b = static_cast<const uint8_t*>(keys)[i]; break;
        }
        out[j] = b;
    }
}

// Forward pass of one row per block (H threads).
__device__ __forceinline__ void mlp_forward_row(const __half* __restrict__ p, const float* __restrict__ x, float* sx,
                                                float* z1, float* h1, float* z2, float* h2, float* y) {
    const int j = threadIdx.x;
    if (j < F) sx[j] = x[j];
    __syncthreads();
    float a = __half2float(p[P_B1 + j]);
    for (int i = 0; i < F; ++i) a += __half2float(p[P_W1 + j * F + i]) * sx[i];
    z1[j] = a;
    h1[j] = a > 0.f ? a : 0.f;
    __syncthreads();
    float b = __half2float(p[P_B2 + j]);
    for (int k = 0; k < H; ++k) b += __half2float(p[P_W2 + j * H + k]) * h1[k];
    z2[j] = b;
    h2[j] = b > 0.f ? b : 0.f;
    __syncthreads();
    if (j < O) {
        float c = __half2float(p[P_B3 + j]);
        for (int k = 0; k < H; ++k) c += __half2float(p[P_W3 + j * H + k]) * h2[k];
        y[j] = c;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(H) k_mlp_forward(const __half* __restrict__ p, const float* __restrict__ x, int rows,
                                                   float* __restrict__ out) {
    __shared__ float sx[F], z1[H], h1[H], z2[H], h2[H], y[O];
    for (int r = blockIdx.x; r < rows; r += gridDim.x) {
        mlp_forward_row(p, x + (size_t)r * F, sx, z1, h1, z2, h2, y);
        if (threadIdx.x < O) out[(size_t)r * O + threadIdx.x] = y[threadIdx.x];
        __syncthreads();
    }
}

// Masked mean-squared error over rows x O outputs; gradients of every
// parameter accumulated per block in shared memory (thread j owns row j of
// W1 / W2 and column j of W3), then added to `grads` once per block.
__global__ void __launch_bounds__(H) k_mlp_fwd_bwd(const __half* __restrict__ p, const float* __restrict__ x,
                                                   const float* __restrict__ tgt, const float* __restrict__ mask,
                                                   int rows, float scale, float* __restrict__ grads,
                                                   float* __restrict__ loss) {
    __shared__ float g[P_TOTAL];
    __shared__ float sx[F], z1[H], h1[H], z2[H], h2[H], y[O], dy[O], dz2[H];
    __shared__ float lsum;
    const int j = threadIdx.x;
    for (int i = j; i < P_TOTAL; i += H) g[i] = 0.f;
    if (j == 0) lsum = 0.f;
    __syncthreads();
    for (int r = blockIdx.x; r < rows; r += gridDim.x) {
        mlp_forward_row(p, x + (size_t)r * F, sx, z1, h1, z2, h2, y);
        if (j < O) {
            float mk = mask[(size_t)r * O + j];
            float e = (y[j] - tgt[(size_t)r * O + j]) * mk;
            dy[j] = 2.f * e * scale;
            atomicAdd(&lsum, e * e * scale);
        }
        __syncthreads();
        if (j < O) g[P_B3 + j] += dy[j];
        float dh2 = 0.f;
        for (int o = 0; o < O; ++o) {
            g[P_W3 + o * H + j] += dy[o] * h2[j];
            dh2 += __half2float(p[P_W3 + o * H + j]) * dy[o];
        }
        float d2 = z2[j] > 0.f ? dh2 : 0.f;
        dz2[j] = d2;
        __syncthreads();
        g[P_B2 + j] += d2;
        for (int k = 0; k < H; ++k) g[P_W2 + j * H + k] += d2 * h1[k];
        float dh1 = 0.f;
        for (int k = 0; k < H; ++k) dh1 += __half2float(p[P_W2 + k * H + j]) * dz2[k];
        float d1 = z1[j] > 0.f ? dh1 : 0.f;
        g[P_B1 + j] += d1;
        for (int i = 0; i < F; ++i) g[P_W1 + j * F + i] += d1 * sx[i];
        __syncthreads();
    }
    for (int i = j; i < P_TOTAL; i += H)
        if (g[i] != 0.f) atomicAdd(&grads[i], g[i]);
    if (j == 0) atomicAdd(loss, lsum);
}

__global__ void k_adam(float* __restrict__ master, __half* __restrict__ p, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, int n, float lr, float c1, float c2) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.f - b1) * gi;
        float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float w = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        master[i] = w;
        p[i] = __float2half_rn(w);
    }
}

struct selector_state {
    std::mutex mu;
    bool loaded = false;
    std::vector<uint16_t> params;
    float mean[F], stdv[F];
    void* dparams[16] = {};
    // Plan features (16..19) of the request lists the weights were trained
    // on, and how far from them the network is trusted; empty: everywhere.
    std::vector<float> support;
    float radius = 0.f;
};
selector_state g_sel;

}  // namespace

// Features 16..19: the aggregation list (cost drivers of every variant's
// per-row work): value bytes read per row, accumulators, float SUMs (64-bit
// shared-memory adds are emulated, several times a 32-bit atomic) and
// MIN / MAX accumulators.
void selector_plan_features(const agg_plan& p, float* f4) {
    f4[0] = (float)((double)p.value_bytes_per_row / 32.0);
    f4[1] = (float)(p.d.n_acc / 8.0);
    f4[2] = (float)(p.d.n_cls[CL_FSUM] / 4.0);
    f4[3] = (float)((p.d.n_cls[CL_MIN] + p.d.n_cls[CL_MAX]) / 8.0);
}

void selector_features(const col& key_in, float* f, cudaStream_t s) {
    owned_col widened;
    col key = key_in;
    if (size_of(key.type) < 4) {
        widened = widen_to_32(key, s);
        key.data = widened.buf.get();
        key.type = widened.type;
    }
    const int64_t n = key.n;
    for (int i = 0; i < F; ++i) f[i] = 0.f;
    if (n == 0) return;
    const int64_t m = std::min<int64_t>(n, GX_SEL_SAMPLE_ROWS);
    const int64_t stride = std::max<int64_t>(1, n / m);
    dbuf samp((size_t)m * 8, s), sorted((size_t)m * 8, s), regs(8192 * 4, s);
    k_sample<<<grid_for(m, 256, 4), 256, 0, s>>>(key.data, size_of(key.type), vkind_of(key.type), m, stride,
                                                   samp.get<unsigned long long>());
    GX_LAUNCHED();
    col sc;
    sc.data = samp.get();
    sc.n = m;
    sc.type = GX_UINT64;
    // Keys of 4 bytes or less are sampled zero-extended: their low 32 bits
    // order them (four 8-bit passes instead of eight).
    radix_sort(sc, nullptr, 0, false, 0, size_of(key.type) == 8 ? -1 : 32, false, sorted.get(), nullptr, nullptr, 0,
               s);
    hll_registers(key, m, stride, regs.get<unsigned>(), s);
    // Pinned host staging (one buffer per host thread, kept): a pageable
    // destination would make the driver bounce the copy through its own.
    struct pinned_sample {
        void* p = nullptr;
        ~pinned_sample() {
            if (p) cudaFreeHost(p);
        }
    };
    static thread_local pinned_sample stage;
    if (!stage.p) GX_CUDA(cudaMallocHost(&stage.p, (size_t)GX_SEL_SAMPLE_ROWS * 8 + 8192 * 4));
    const uint64_t* h = static_cast<const uint64_t*>(stage.p);
    const unsigned* hr = reinterpret_cast<const unsigned*>(static_cast<char*>(stage.p) + (size_t)GX_SEL_SAMPLE_ROWS * 8);
    GX_CUDA(cudaMemcpyAsync(stage.p, sorted.get(), (size_t)m * 8, cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaMemcpyAsync(static_cast<char*>(stage.p) + (size_t)GX_SEL_SAMPLE_ROWS * 8, regs.get(), 8192 * 4,
                            cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaStreamSynchronize(s));
    // Runs of equal keys in the sorted sample: their count, the singletons
    // and the eight longest (kept in order while scanning; the device waits
    // for this, so no full sort of ~m run lengths).
    int64_t top[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t f1 = 0, nruns = 0;
    for (int64_t i = 0; i < m;) {
        int64_t j = i + 1;
        while (j < m && h[j] == h[i]) ++j;
        const int64_t len = j - i;
        ++nruns;
        f1 += len == 1;
        if (len > top[7]) {
            int t = 7;
            while (t > 0 && top[t - 1] < len) {
                top[t] = top[t - 1];
                --t;
            }
            top[t] = len;
        }
        i = j;
    }
    const double d = (double)nruns;
    const double hll = hll_estimate(hr);
    const double gee = std::sqrt((double)n / (double)m) * (double)f1 + (d - (double)f1);
    f[0] = (float)(std::log2((double)n) / 28.0);
    f[1] = size_of(key.type) == 8 ? 1.f : 0.f;
    f[2] = (float)(std::log2(1.0 + hll) / 14.0);
    f[3] = (float)(std::log2(1.0 + d) / 14.0);
    f[4] = (float)(d / (double)m);
    f[5] = (float)((double)f1 / (double)m);
    for (int t = 0; t < 8; ++t) f[6 + t] = (float)((double)top[t] / (double)m);
    f[14] = (float)(std::log2(1.0 + gee) / 28.0);
    f[15] = (float)(std::log2((double)n / std::max(1.0, gee)) / 28.0);
}

int64_t selector_param_count() { return P_TOTAL; }

void selector_load(const uint16_t* params, const float* mean, const float* stdv) {
    std::lock_guard<std::mutex> g(g_sel.mu);
    g_sel.params.assign(params, params + P_TOTAL);
    for (int i = 0; i < F; ++i) {
        g_sel.mean[i] = mean ? mean[i] : 0.f;
        g_sel.stdv[i] = stdv && stdv[i] > 0.f ? stdv[i] : 1.f;
    }
    for (auto& p : g_sel.dparams) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    g_sel.loaded = true;
}

bool selector_loaded() {
    std::lock_guard<std::mutex> g(g_sel.mu);
    return g_sel.loaded;
}

void selector_set_plan_support(const float* f4, int count, float radius) {
    std::lock_guard<std::mutex> g(g_sel.mu);
    g_sel.support.assign(f4, f4 + (size_t)count * (F - GX_SEL_KEY_FEATURES));
    g_sel.radius = radius;
}

// Whether the network has seen a request list like this one: plan features
// within the radius (largest coordinate difference) of a registered one.
static bool plan_in_support(const float* f4) {
    constexpr int PF = F - GX_SEL_KEY_FEATURES;
    std::lock_guard<std::mutex> g(g_sel.mu);
    if (g_sel.support.empty()) return true;
    for (size_t b = 0; b < g_sel.support.size(); b += PF) {
        float d = 0.f;
        for (int i = 0; i < PF; ++i) d = std::max(d, std::fabs(f4[i] - g_sel.support[b + i]));
        if (d <= g_sel.radius) return true;
    }
    return false;
}

static const __half* selector_device_params() {
    int d = dev().device;
    std::lock_guard<std::mutex> g(g_sel.mu);
    if (!g_sel.loaded) return nullptr;
    if (!g_sel.dparams[d]) {
        void* p = nullptr;
        GX_CUDA(cudaMalloc(&p, P_TOTAL * 2));
        GX_CUDA(cudaMemcpy(p, g_sel.params.data(), P_TOTAL * 2, cudaMemcpyHostToDevice));
        g_sel.dparams[d] = p;
    }
    return static_cast<const __half*>(g_sel.dparams[d]);
}

void mlp_forward(const void* params, const float* x, int rows, float* out, cudaStream_t s) {
    if (rows <= 0) return;
    k_mlp_forward<<<std::min(rows, dev().sm_count * 8), H, 0, s>>>(static_cast<const __half*>(params), x, rows, out);
    GX_LAUNCHED();
}

void mlp_forward_backward(const void* params, const float* x, const float* tgt, const float* mask, int rows,
                          float* grads, float* loss, cudaStream_t s) {
    GX_CUDA(cudaMemsetAsync(grads, 0, P_TOTAL * sizeof(float), s));
    GX_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), s));
    if (rows <= 0) return;
    float scale = 1.f / (float)((int64_t)rows * O);
    k_mlp_fwd_bwd<<<std::min(rows, dev().sm_count * 2), H, 0, s>>>(static_cast<const __half*>(params), x, tgt, mask,
                                                                    rows, scale, grads, loss);
    GX_LAUNCHED();
}

void mlp_adam(float* master, void* params, const float* grads, float* m, float* v, int step, float lr,
              cudaStream_t s) {
    float c1 = 1.f - std::pow(0.9f, (float)step), c2 = 1.f - std::pow(0.999f, (float)step);
    k_adam<<<grid_for(P_TOTAL, 256, 1), 256, 0, s>>>(master, static_cast<__half*>(params), grads, m, v, P_TOTAL, lr,
                                                      c1, c2);
    GX_LAUNCHED();
}

void selector_predict(const float* feats, int rows, float* scores, cudaStream_t s) {
    const __half* p = selector_device_params();
    require(p != nullptr, "selector: no weights loaded (gx_selector_load)");
    std::vector<float> xs((size_t)rows * F);
    for (int r = 0; r < rows; ++r)
        for (int i = 0; i < F; ++i)
            xs[(size_t)r * F + i] = (feats[(size_t)r * F + i] - g_sel.mean[i]) / g_sel.stdv[i];
    dbuf dx(xs.size() * 4, s), dout((size_t)rows * O * 4, s);
    GX_CUDA(cudaMemcpyAsync(dx.get(), xs.data(), xs.size() * 4, cudaMemcpyHostToDevice, s));
    mlp_forward(p, dx.get<float>(), rows, dout.get<float>(), s);
    GX_CUDA(cudaMemcpyAsync(scores, dout.get(), (size_t)rows * O * 4, cudaMemcpyDeviceToHost, s));
    GX_CUDA(cudaStreamSynchronize(s));
}

// AUTO with the learned selector; falls back to the reference's NDV rule
// when no weights are loaded or the request list is outside the support
// registered with the weights.
int selector_choose(const col& key, const agg_plan& plan, int* radix_bits, cudaStream_t s) {
    *radix_bits = 0;
    float pf[F - GX_SEL_KEY_FEATURES];
    selector_plan_features(plan, pf);
    // No weights, or a request list unlike those the weights were trained
    // on (the network's scores there are extrapolations): the plain rule.
    if (!selector_loaded() || !plan_in_support(pf)) {
        int64_t est = ndv_estimate(key, s);
        return est <= (size_of(key.type) == 4 ? (1 << 14) : (1 << 18)) ? GX_GB_HASH : GX_GB_PARTITION;
    }
    float f[F], y[O];
    selector_features(key, f, s);
    std::copy(pf, pf + (F - GX_SEL_KEY_FEATURES), f + GX_SEL_KEY_FEATURES);
    selector_predict(f, 1, y, s);
    static const int variants[3] = {GX_GB_HASH, GX_GB_SORT, GX_GB_PARTITION};
    int best = 0;
    for (int v = 1; v < GX_SEL_NUM_VARIANTS; ++v)
        if (y[v] < y[best]) best = v;
    if (variants[best] == GX_GB_PARTITION) {
        int bf = 0;
        for (int k = 1; k < GX_SEL_NUM_FANOUTS; ++k)
            if (y[GX_SEL_NUM_VARIANTS + k] < y[GX_SEL_NUM_VARIANTS + bf]) bf = k;
        // The fan-out head overrides the engine's own rule (radix bits from
        // the group estimate) only for a predicted gain of at least 20% over
        // one 8-bit pass: a second radix pass costs a full extra scatter, so a
        // near-tie is not worth the risk of a misprediction.
        const float gain = y[GX_SEL_NUM_VARIANTS] - y[GX_SEL_NUM_VARIANTS + bf];  // log2 time
        *radix_bits = (bf == 0 || gain >= 0.263f) ? FANOUT_BITS[bf] : 0;
    }
    return variants[best];
}

}  // namespace gx
