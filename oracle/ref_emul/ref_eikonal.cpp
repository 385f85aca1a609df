// Host build of the reference's eikonal `Update` kernel (Update.h with the
// Isotropic_.h or Riemann_.h model), driven by a restatement of the reference's
// host loops.  TEST INFRASTRUCTURE: used only to generate golden fixtures and to
// pin the oracle; never linked by the product.
//
// Compile-time configuration (set by oracle/ref_emul/Makefile):
//   AGDREF_ISO (0|1), AGDREF_DIAG (0|1: the Diagonal model, Isotropic_.h with
//   per-point squared dual costs as geometry, _SetGeometry.py:134-135), AGDREF_NDIM, AGDREF_SHAPE_I (comma list), AGDREF_SIZE_I,
//   AGDREF_LOG2_SIZE_I, AGDREF_NITER_I, AGDREF_MULTIP (0|1), AGDREF_FLOW (0|1),
//   AGDREF_FACTOR (0|1, source factorisation, factor_macro of _Kernel.py:47-49),
//   AGDREF_ORDER2 (0|1, second order scheme, order2_macro of _Kernel.py:51-54),
//   AGDREF_WALLS (0|1, obstacles, walls_macro of _Kernel.py:111),
//   AGDREF_DRIFT (0|1, the Rander model: Riemann_.h with a drift, _Kernel.py:58-59).
//
// The block below states the same compile-time traits that the reference's
// `cupy_module_helper.traits_header` emits for these models
// (agd/Eikonal/HFM_CUDA/_Kernel.py:23-92, 94-160; kernel_traits.py:6-117).
#include "cuda_host_shim.h"
#include <cstring>
#include <vector>

#ifndef AGDREF_FACTOR
#define AGDREF_FACTOR 0
#endif
#if AGDREF_FACTOR
#define factor_macro true
#endif
#ifndef AGDREF_ORDER2
#define AGDREF_ORDER2 0
#endif
#if AGDREF_ORDER2
#define order2_macro true
#endif
#ifndef AGDREF_WALLS
#define AGDREF_WALLS 0
#endif
#define pruning_macro false
#define geom_first_macro true
typedef float Scalar;
#define Scalar_macro
typedef int Int;
#define Int_macro
const Int Int_Max = 2147483647;
typedef int OffsetT;
#define OffsetT_macro
const int shape_i[AGDREF_NDIM] = {AGDREF_SHAPE_I};
const int niter_i = AGDREF_FLOW ? 1 : AGDREF_NITER_I;
#define multiprecision_macro AGDREF_MULTIP
#if AGDREF_MULTIP
#define strict_iter_o_macro true
#define strict_iter_i_macro true
#endif
#define ndim_macro AGDREF_NDIM
#if AGDREF_FLOW
#define fim_macro false
#define flow_weights_macro true
#define flow_weightsum_macro true
#define flow_indices_macro true
#define flow_vector_macro true
#else
#define fim_macro true
#endif
#define import_scheme_macro false
#define local_i_macro true
#define periodic_macro false
#define isotropic_macro AGDREF_ISO
#define walls_macro AGDREF_WALLS
#ifndef AGDREF_DIAG
#define AGDREF_DIAG 0
#endif
#ifndef AGDREF_DRIFT
#define AGDREF_DRIFT 0
#endif
#if AGDREF_DRIFT
#define drift_macro 1
#endif
#if AGDREF_ISO
#define geom_indep_macro AGDREF_NDIM
#elif AGDREF_DIAG
#define geom_indep_macro 0
#define geom_size_macro AGDREF_NDIM
#else
#define geom_indep_macro 0
#define geom_size_macro ((AGDREF_NDIM * (AGDREF_NDIM + 1)) / 2 + (AGDREF_DRIFT ? AGDREF_NDIM : 0))
#endif
#define hfm_debug_macro false
const int size_i = AGDREF_SIZE_I;
const int log2_size_i = AGDREF_LOG2_SIZE_I;

// The reference's module constant `atol` would collide with the C library's atol().
#define atol agdref_atol
#if AGDREF_ISO || AGDREF_DIAG
#include "Isotropic_.h"
#else
// Riemann_.h includes EuclideanFactor.h inside a FACTOR(...) macro argument, which
// NVRTC accepts and g++ rejects; including it (and its prerequisites) beforehand
// turns that nested include into a no-op under #pragma once.
#include "TypeTraits.h"
#include "EuclideanFactor.h"
#include "Riemann_.h"
#endif

namespace {

struct Args {
    Scalar *u, *uNext;
    Int *uq, *uqNext;
    const Scalar *geom;
    const BoolPack *seeds;
    const Scalar *rhs;
    Scalar *fw, *fws, *fv;
    Int *fi;
    Int *list;
    BoolAtom *scorePrev, *scoreNext, *updateNext;
};

#if AGDREF_WALLS
const WallT *g_wall_dist = nullptr;  // wallDist of the next solves (tile layout)
#endif

void thunk(void *p) {
    Args &a = *static_cast<Args *>(p);
    (void)a;
    Update(
#if AGDREF_MULTIP
        a.u, a.uq, a.uNext, a.uqNext,
#else
        a.u,
#endif
        a.geom, a.seeds, a.rhs,
#if AGDREF_WALLS
        g_wall_dist,
#endif
#if AGDREF_FLOW
        a.fw, a.fws, a.fi, a.fv, a.list, a.updateNext
#else
        a.list, a.scorePrev, a.scoreNext, a.updateNext
#endif
    );
}

void set_common(const int *shape, float atol_, float rtol_, const float *iso_w, float mstep,
                float mmax, int *size_o_out, int *size_tot_out) {
    int so = 1;
    for (int k = 0; k < ndim; ++k) {
        shape_tot[k] = shape[k];
        shape_o[k] = (shape[k] + shape_i[k] - 1) / shape_i[k];
        so *= shape_o[k];
    }
    size_o = so;
    size_tot = so * size_i;
#if geom_indep_macro
    size_geom_o = 1;
    size_geom_i = 1;
    size_geom_tot = 1;
#else
    size_geom_tot = size_tot;
#endif
    atol = atol_;
    rtol = rtol_;
#if AGDREF_ISO
    for (int k = 0; k < ndim; ++k) weights[k] = iso_w[k];
#else
    (void)iso_w;
#endif
#if AGDREF_MULTIP
    multip_step = mstep;
    multip_max = mmax;
#else
    (void)mstep;
    (void)mmax;
#endif
    *size_o_out = size_o;
    *size_tot_out = size_tot;
}

}  // namespace

extern "C" {

#if AGDREF_FACTOR
// The module constants of source factorisation (_Kernel.py:301-308).
void agdref_set_factor(const float *origin, float radius2, const float *metric) {
    for (int k = 0; k < ndim; ++k) factor_origin[k] = origin[k];
    factor_radius2 = radius2;
    for (int k = 0; k < factor_size; ++k) factor_metric[k] = metric[k];
}
#endif

#if AGDREF_WALLS
// The wallDist argument of the next Update calls (_SetGeometry.py:262-280).
void agdref_set_walls(const unsigned char *wall_dist) { g_wall_dist = wall_dist; }
#endif

#if AGDREF_ORDER2
// The module constant of the second order scheme (_Kernel.py:310-314).
void agdref_set_order2(float threshold) { order2_threshold = threshold; }
#endif

#if !AGDREF_FLOW
// Restatement of _solvers.fast_iterative_method (agd/Eikonal/HFM_CUDA/_solvers.py:94-120),
// with the stop test of _StopCriterion.InitStop (np.any(update_o)), and the
// values/valuesNext swap of _solvers.KernelArgs for strict_iter_o.
// `values`/`valuesq` hold the initial state and receive the final one.
// Returns niter_o; `nupdate_tiles` receives the number of tile visits.
int agdref_fim_solve(const int *shape, float atol_, float rtol_, int front_width,
                     const float *iso_w, float mstep, float mmax, float *values, int *valuesq,
                     const float *geom, const unsigned char *seedTags, const float *rhs,
                     const unsigned char *trigger_o, int nitermax, long long *nupdate_tiles) {
    int so, st;
    set_common(shape, atol_, rtol_, iso_w, mstep, mmax, &so, &st);
    fim_front_width = (BoolAtom)front_width;
    std::vector<BoolAtom> updateNext(trigger_o, trigger_o + so), scoreA(so, 0), scoreB(so, 0);
    BoolAtom *scorePrev = scoreA.data(), *scoreNext = scoreB.data();
    std::vector<Int> list;
#if AGDREF_MULTIP
    std::vector<Scalar> u2(values, values + st);
    std::vector<Int> uq2(valuesq, valuesq + st);
    Scalar *ucur = values, *unext = u2.data();
    Int *uqcur = valuesq, *uqnext = uq2.data();
#endif
    long long visits = 0;
    int niter = 0;
    for (; niter < nitermax; ++niter) {
        list.clear();
        for (int n = 0; n < so; ++n)
            if (updateNext[n]) list.push_back(n);
        if (list.empty()) break;
        std::swap(scorePrev, scoreNext);
        std::fill(updateNext.begin(), updateNext.end(), 0);
        std::fill(scoreNext, scoreNext + so, 0);
        Args a{};
#if AGDREF_MULTIP
        a.u = ucur; a.uq = uqcur; a.uNext = unext; a.uqNext = uqnext;
#else
        a.u = values;
#endif
        a.geom = geom; a.seeds = seedTags; a.rhs = rhs;
        a.list = list.data(); a.scorePrev = scorePrev; a.scoreNext = scoreNext;
        a.updateNext = updateNext.data();
        for (size_t b = 0; b < list.size(); ++b) agdref_run_block(thunk, &a, size_i, (int)b);
        visits += (long long)list.size();
#if AGDREF_MULTIP
        std::swap(ucur, unext);
        std::swap(uqcur, uqnext);
#endif
    }
#if AGDREF_MULTIP
    if (ucur != values) {
        std::memcpy(values, ucur, sizeof(Scalar) * st);
        std::memcpy(valuesq, uqcur, sizeof(Int) * st);
    }
#endif
    if (nupdate_tiles) *nupdate_tiles = visits;
    return niter;
}
#else
// One global iteration of the flow variant of `Update` (_PostProcess.PostProcess,
// agd/Eikonal/HFM_CUDA/_PostProcess.py:46-95, with atol=inf, rtol=0 and
// nitermax_o=1), exporting flow_weights, flow_weightsum, flow_indices, flow_vector.
// With multiprecision the refreshed values land in values/valuesq (KernelArgs swap).
int agdref_flow(const int *shape, const float *iso_w, float mstep, float mmax, float *values,
                int *valuesq, const float *geom, const unsigned char *seedTags, const float *rhs,
                float *flow_weights, float *flow_weightsum, int *flow_indices,
                float *flow_vector) {
    int so, st;
    set_common(shape, INFINITY, 0.f, iso_w, mstep, mmax, &so, &st);
    std::vector<Int> list(so);
    for (int n = 0; n < so; ++n) list[n] = n;
    std::vector<BoolAtom> updateNext(so, 0);
    Args a{};
#if AGDREF_MULTIP
    std::vector<Scalar> u2(values, values + st);
    std::vector<Int> uq2(valuesq, valuesq + st);
    a.u = values; a.uq = valuesq; a.uNext = u2.data(); a.uqNext = uq2.data();
#else
    a.u = values;
#endif
    a.geom = geom; a.seeds = seedTags; a.rhs = rhs;
    a.fw = flow_weights; a.fws = flow_weightsum; a.fi = flow_indices; a.fv = flow_vector;
    a.list = list.data(); a.updateNext = updateNext.data();
    for (int b = 0; b < so; ++b) agdref_run_block(thunk, &a, size_i, b);
#if AGDREF_MULTIP
    std::memcpy(values, u2.data(), sizeof(Scalar) * st);
    std::memcpy(valuesq, uq2.data(), sizeof(Int) * st);
#endif
    return 0;
}
#endif

// Direct access to the reference's per-point Selling decomposition
// (Geometry2.h:21-48 / Geometry3.h:22-58, via Riemann_.h:23-29) for golden vectors.
#if !AGDREF_ISO && !AGDREF_DIAG && !AGDREF_DRIFT && !AGDREF_FLOW && !AGDREF_MULTIP
void agdref_selling(const float *m, int n, float *w, int *e) {
    for (int p = 0; p < n; ++p) {
        Scalar wl[symdim];
        OffsetT el[symdim][ndim];
        decomp_m(m + symdim * p, wl, el);
        for (int r = 0; r < symdim; ++r) {
            w[symdim * p + r] = wl[r];
            for (int j = 0; j < ndim; ++j) e[(symdim * p + r) * ndim + j] = el[r][j];
        }
    }
}
#endif
}
