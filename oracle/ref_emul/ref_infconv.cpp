// Host build of the reference's inf-convolution kernel (Kernel_InfConvolution.h) with
// the traits used for the geodesic 'eucl' map: uint8, 3^d kernel, min-plus,
// upper saturation at 255 (_GetGeodesics.py:51-75; inf_convolution.py:32-93).
// TEST INFRASTRUCTURE only.
#include "cuda_host_shim.h"

typedef unsigned char T;
#define T_macro
#if AGDREF_NDIM == 2
const int shape_c[2] = {3, 3};
const int size_c = 9;
#else
const int shape_c[3] = {3, 3, 3};
const int size_c = 27;
#endif
#define mix_is_min_macro 1
const int ndim = AGDREF_NDIM;
#define upper_saturation_macro 1
const unsigned char T_Sup = 255;
const unsigned char T_Inf = 0;
#define hfm_debug_macro false

#include "Kernel_InfConvolution.h"

extern "C" {
// niter launches of InfConvolution, ping-ponging between arr and out
// (inf_convolution.py:87-91).  Returns a pointer to whichever buffer holds the result.
const unsigned char *agdref_infconv(const int *shape, const unsigned char *kernel, int niter,
                                    unsigned char *arr, unsigned char *out) {
    int st = 1;
    for (int k = 0; k < ndim; ++k) {
        shape_tot[k] = shape[k];
        st *= shape[k];
    }
    size_tot = st;
    for (int i = 0; i < size_c; ++i) kernel_c[i] = kernel[i];
    const int bs = 1024;
    blockDim.x = bs;
    for (int it = 0; it < niter; ++it) {
        for (int t = 0; t < st; ++t) {
            blockIdx.x = t / bs;
            threadIdx.x = t % bs;
            InfConvolution(arr, out);
        }
        unsigned char *tmp = arr; arr = out; out = tmp;
    }
    return arr;
}
}
