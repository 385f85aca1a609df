#include "agd_internal.h"
using namespace agd;
extern "C" {
int agd_eucl_map(int, const int *, const uint8_t *, int, int, uint8_t *, uint8_t *, agd_stream_t) {
    return set_error(AGD_STATUS_UNSUPPORTED, "not built");
}
int agd_geodesics(const agd_instance *, const float *, const float *, const uint8_t *, const float *, int, float,
                  float, int, int, int, int, float *, int, int32_t *, int8_t *, agd_stream_t) {
    return set_error(AGD_STATUS_UNSUPPORTED, "not built");
}
}
