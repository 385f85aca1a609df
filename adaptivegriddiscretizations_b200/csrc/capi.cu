// Error reporting and version of the C ABI (include/agd_b200.h).
#include <cstdio>
#include <cstring>

#include "agd_internal.h"

namespace agd {

static thread_local char g_msg[512] = "";

void clear_error() { g_msg[0] = 0; }

int set_error(int status, const char *msg) {
    std::snprintf(g_msg, sizeof(g_msg), "%s", msg);
    return status;
}

int set_cuda_error(const char *what, cudaError_t err) {
    std::snprintf(g_msg, sizeof(g_msg), "%s: %s (%s)", what, cudaGetErrorName(err), cudaGetErrorString(err));
    return AGD_STATUS_CUDA;
}

}  // namespace agd

extern "C" {
const char *agd_last_error(void) { return agd::g_msg; }
int agd_version(void) { return 4; }
}
