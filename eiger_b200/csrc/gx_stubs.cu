// gx_stubs.cu — entry points whose implementation lands in later files.
#include "gx_groupby.h"

extern "C" {
gx_status gx_batch_plan_create(const gx_batch_instance*, int32_t, int64_t, gx_stream_t, gx_batch_plan**) { return GX_EUNSUPPORTED; }
gx_status gx_batch_run(gx_batch_plan*, gx_stream_t) { return GX_EUNSUPPORTED; }
gx_status gx_batch_run_per_instance(gx_batch_plan*, gx_stream_t) { return GX_EUNSUPPORTED; }
gx_status gx_batch_results(const gx_batch_plan*, gx_batch_result*) { return GX_EUNSUPPORTED; }
gx_status gx_batch_tuning(const gx_batch_plan*, int32_t*, int32_t*) { return GX_EUNSUPPORTED; }
void gx_batch_plan_free(gx_batch_plan*) {}
gx_status gx_dictionary_encode_strings(gx_column_view, int64_t, gx_stream_t, gx_column*, int64_t*) { return GX_EUNSUPPORTED; }
}
