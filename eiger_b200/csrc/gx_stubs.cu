// gx_stubs.cu — entry points whose implementation lands in later files.
#include "gx_groupby.h"

extern "C" {
gx_status gx_dictionary_encode_strings(gx_column_view, int64_t, gx_stream_t, gx_column*, int64_t*) { return GX_EUNSUPPORTED; }
}
