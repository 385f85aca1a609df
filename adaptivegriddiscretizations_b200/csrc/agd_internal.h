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
    // Offset of that stencil in the workspace's stencil region, in floats (-1:
    // none); the host sets `stencil` from it once the workspace is known.
    long long stencil_off;
};

// Thread-local error message for agd_last_error().
void clear_error();
int set_error(int status, const char *msg);
int set_cuda_error(const char *what, cudaError_t err = cudaGetLastError());

// Min-plus distance map in grid layout (geodesic.cu): 0 at the mask points,
// `npasses` passes of the 3^ndim kernel round(5 |o|) (l1 false) or |o|_1 (l1
// true), saturated at 255, values above `cut` set to 255; nb instances one
// after the other, each its own map.  tmp: nb prod(shape) bytes.
int distance_map(int ndim, const int *shape, const uint8_t *mask, int npasses, int cut, bool l1, uint8_t *out,
                 uint8_t *tmp, cudaStream_t st, int nb = 1);

}  // namespace agd
