#include "agd_internal.h"
using namespace agd;
extern "C" {
size_t agd_reverse_workspace_bytes(const agd_instance *) { return 0; }
int agd_reverse(const agd_instance *, const float *, const int32_t *, const float *, const float *, float *, float,
                float, void *, size_t, agd_stats *, const agd_launch *, agd_stream_t) {
    return set_error(AGD_STATUS_UNSUPPORTED, "not built");
}
}
