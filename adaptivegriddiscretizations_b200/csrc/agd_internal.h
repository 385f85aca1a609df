// Internal host/device declarations shared by the .cu files of libagd_b200.
#pragma once
#include <cuda_runtime.h>

#include "../../include/agd_b200.h"

namespace agd {

// An agd_instance with the quantities derived from it (device copy per instance).
struct Inst {
    agd_instance a;
    int shape_o[3];
    int size_o;
    int size_i;
    long long size_tot;
    int tile_base;  // first global tile id of this instance in a batched launch
    int variant;    // compiled tile-visit variant, -1 if none
    // Riemann models: per-point Selling stencil computed once per solve (weights,
    // then packed offsets, symdim planes each, tile layout), or null to compute
    // it at every visit.
    float *stencil;
};

// Thread-local error message for agd_last_error().
void clear_error();
int set_error(int status, const char *msg);
int set_cuda_error(const char *what, cudaError_t err = cudaGetLastError());

}  // namespace agd
