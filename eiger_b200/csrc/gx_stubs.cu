// gx_stubs.cu — entry points whose implementation lands in later files.
#include "gx_groupby.h"

namespace gx {
int selector_choose(const col& key, int* radix_bits, cudaStream_t s) {
    *radix_bits = 0;
    int64_t est = ndv_estimate(key, s);
    return est <= (size_of(key.type) == 4 ? (1 << 14) : (1 << 18)) ? GX_GB_HASH : GX_GB_PARTITION;
}
}  // namespace gx

extern "C" {
gx_status gx_dictionary_encode_strings(gx_column_view, int64_t, gx_stream_t, gx_column*, int64_t*) { return GX_EUNSUPPORTED; }
gx_status gx_selector_features(gx_column_view, gx_stream_t, float*) { return GX_EUNSUPPORTED; }
int64_t gx_selector_param_count(void) { return 0; }
gx_status gx_selector_load(const uint16_t*, const float*, const float*) { return GX_EUNSUPPORTED; }
gx_status gx_selector_predict(const float*, int32_t, float*) { return GX_EUNSUPPORTED; }
gx_status gx_mlp_forward(const void*, const float*, int32_t, float*, gx_stream_t) { return GX_EUNSUPPORTED; }
gx_status gx_mlp_forward_backward(const void*, const float*, const float*, const float*, int32_t, float*, float*, gx_stream_t) { return GX_EUNSUPPORTED; }
gx_status gx_mlp_adam_step(float*, void*, const float*, float*, float*, int32_t, float, gx_stream_t) { return GX_EUNSUPPORTED; }
gx_status gx_batch_plan_create(const gx_batch_instance*, int32_t, int64_t, gx_stream_t, gx_batch_plan**) { return GX_EUNSUPPORTED; }
gx_status gx_batch_run(gx_batch_plan*, gx_stream_t) { return GX_EUNSUPPORTED; }
gx_status gx_batch_run_per_instance(gx_batch_plan*, gx_stream_t) { return GX_EUNSUPPORTED; }
gx_status gx_batch_results(const gx_batch_plan*, gx_batch_result*) { return GX_EUNSUPPORTED; }
gx_status gx_batch_tuning(const gx_batch_plan*, int32_t*, int32_t*) { return GX_EUNSUPPORTED; }
void gx_batch_plan_free(gx_batch_plan*) {}
}
