// Host build of the reference's linear update kernel (Kernel_LinearUpdate.h), used
// for the forward/reverse automatic differentiation systems, driven by a restatement
// of the non-pruning AGSI loop.  TEST INFRASTRUCTURE only.
// Traits as emitted by _PostProcess.SolveLinear (agd/Eikonal/HFM_CUDA/_PostProcess.py:97-152).
#include "cuda_host_shim.h"
#include <vector>

const int shape_i[AGDREF_NDIM] = {AGDREF_SHAPE_I};
const int niter_i = AGDREF_NITER_I;
#define pruning_macro false
const int ndim = AGDREF_NDIM;
const int nrhs = 1;
const int nindex = AGDREF_NINDEX;
#define hfm_debug_macro false
const int size_i = AGDREF_SIZE_I;
const int log2_size_i = AGDREF_LOG2_SIZE_I;

#define atol agdref_atol
#include "Kernel_LinearUpdate.h"

namespace {
struct Args {
    Scalar *u;
    const Scalar *rhs, *diag, *w;
    const Int *idx;
    Int *list;
    BoolAtom *updateNext;
};
void thunk(void *p) {
    Args &a = *static_cast<Args *>(p);
    Update(a.u, a.rhs, a.diag, a.idx, a.w, a.list, a.updateNext);
}
}  // namespace

extern "C" {
// Restatement of _solvers.adaptive_gauss_siedel_iteration without pruning
// (agd/Eikonal/HFM_CUDA/_solvers.py:122-193).  `sol` starts at +inf (unvisited)
// and receives the solution.  Arrays have nindex planes of size_tot entries.
int agdref_linear_solve(const int *shape_o_, float atol_, float rtol_, float *sol,
                        const float *rhs, const float *diag, const int *indices,
                        const float *weights, const unsigned char *trigger_o, int nitermax) {
    int so = 1;
    for (int k = 0; k < ndim; ++k) {
        shape_o[k] = shape_o_[k];
        so *= shape_o_[k];
    }
    size_o = so;
    size_tot = so * size_i;
    atol = atol_;
    rtol = rtol_;
    std::vector<BoolAtom> update(trigger_o, trigger_o + so);
    std::vector<Int> list;
    int niter = 0;
    for (; niter < nitermax; ++niter) {
        list.clear();
        for (int n = 0; n < so; ++n)
            if (update[n]) list.push_back(n);
        if (list.empty()) break;
        std::fill(update.begin(), update.end(), 0);
        Args a{sol, rhs, diag, weights, indices, list.data(), update.data()};
        for (size_t b = 0; b < list.size(); ++b) agdref_run_block(thunk, &a, size_i, (int)b);
    }
    return niter;
}
int agdref_nindex() { return nindex; }
}
