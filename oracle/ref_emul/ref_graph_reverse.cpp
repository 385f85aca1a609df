// Host build of the reference's weighted graph transposition kernel (GraphReverse.h).
// TEST INFRASTRUCTURE only.  Traits as emitted by graph_reverse.py:23-48 (irevT=int8).
#include "cuda_host_shim.h"

typedef int Int;
#define Int_macro
const Int Int_Max = 2147483647;
typedef float weightT;
#define weightT_macro
typedef signed char irevT;
#define irevT_macro
const signed char irevT_Max = 127;
const int invalid = 2147483647;
#define invalid_macro true
#define hfm_debug_macro false

#include "GraphReverse.h"

extern "C" {
// One launch of GraphReverse over size_tot threads (graph_reverse.py:66-77 loops it).
void agdref_graph_reverse_launch(int size_tot_, int nfwd_, int nrev_, const int *fwd, int *rev,
                                 signed char *irev, const float *fwd_weight, float *rev_weight) {
    size_tot = size_tot_;
    nfwd = nfwd_;
    nrev = nrev_;
    const int bs = 1024;
    blockDim.x = bs;
    for (int t = 0; t < size_tot_; ++t) {
        blockIdx.x = t / bs;
        threadIdx.x = t % bs;
        GraphReverse(fwd, rev, irev, fwd_weight, rev_weight);
    }
}
}
