// Host build of the reference's geodesic backtracking kernel (Kernel_GeodesicODE.h,
// precomputed-flow variant of GeodesicODE_Opt.h).  TEST INFRASTRUCTURE only.
// Traits as emitted by the reference for its 'geodesic' kernel
// (agd/Eikonal/HFM_CUDA/_Kernel.py:163-203).  One emulated thread per geodesic; the
// kernel has no block barrier, so threads simply run one after the other.
#include "cuda_host_shim.h"

typedef float Scalar;
#define Scalar_macro
typedef int Int;
#define Int_macro
const Int Int_Max = 2147483647;
typedef int OffsetT;
#define OffsetT_macro
#define pruning_macro false
#define geom_first_macro true
const int shape_i[AGDREF_NDIM] = {AGDREF_SHAPE_I};
const int niter_i = 1;
#define multiprecision_macro false
#define ndim_macro AGDREF_NDIM
#define fim_macro false
#ifndef AGDREF_EUCL_DELAY
#define AGDREF_EUCL_DELAY (AGDREF_NDIM == 2 ? 5 : 6)      // int(sqrt(ndim)/0.25)
#endif
#ifndef AGDREF_NYMIN_DELAY
#define AGDREF_NYMIN_DELAY (AGDREF_NDIM == 2 ? 45 : 55)   // int(8*sqrt(ndim)/0.25)
#endif
const int eucl_delay = AGDREF_EUCL_DELAY;
const int nymin_delay = AGDREF_NYMIN_DELAY;
typedef unsigned char EuclT;
#define EuclT_macro
const unsigned char EuclT_Max = 255;
const int EuclT_Chart = 254;
#define online_flow_macro false
#define chart_macro false
#define flow_vector_macro true
#define local_i_macro false
#define mixed_state_macro false
#define periodic_macro false
#define hfm_debug_macro false
const int size_i = AGDREF_SIZE_I;

#include "Kernel_GeodesicODE.h"

extern "C" {
// One launch of GeodesicODE over nGeo geodesics (one chunk of _GetGeodesics.py:111-134).
void agdref_geodesic_chunk(const int *shape, int nGeo, int max_len_, int pastseed_delay_,
                           float causalityTolerance_, float step, const float *u,
                           const float *flow_vector, const float *flow_weightsum,
                           const unsigned char *eucl, float *x_s, int *len_s, signed char *stop_s) {
    int so = 1;
    for (int k = 0; k < ndim; ++k) {
        shape_tot[k] = shape[k];
        shape_o[k] = (shape[k] + shape_i[k] - 1) / shape_i[k];
        so *= shape_o[k];
    }
    size_tot = so * size_i;
    nGeodesics = nGeo;
    max_len = max_len_;
    pastseed_delay = pastseed_delay_;
    causalityTolerance = causalityTolerance_;
    geodesicStep = step;
    const int bs = 32;
    blockDim.x = bs;
    for (int tid = 0; tid < nGeo; ++tid) {
        blockIdx.x = tid / bs;
        threadIdx.x = tid % bs;
        GeodesicODE(u, flow_vector, flow_weightsum, eucl, x_s, len_s, (ODEStopT *)stop_s);
    }
}
}
