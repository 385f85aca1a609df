// Shared device code of the B200 eikonal path: tile geometry, Selling's
// decomposition, the eikonal update operator, and the bounded grid barrier used
// by the persistent kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/agd_b200.h"

namespace agd {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kIntMax = 2147483647;

__device__ __forceinline__ float finf() { return __int_as_float(0x7f800000); }

// ------------------------------------------------------------------ tiles ---
// A tile ("block" in the reference) of S0 x S1 (x S2) points; the bilevel index
// of a point is n_t = n_o * SIZE + n_i (agd/FiniteDifferences.py:164-222,
// cuda/Grid.h:15-35), with row-major n_o over tiles and n_i inside the tile.
template <int D_, int S0_, int S1_, int S2_>
struct Tile {
    static constexpr int D = D_, S0 = S0_, S1 = S1_, S2 = (D_ == 3 ? S2_ : 1);
    static constexpr int SIZE = S0 * S1 * S2;
    static constexpr int P = SIZE / 32;  // points per lane (one warp per tile)
    static_assert(SIZE % 32 == 0, "tile size must be a multiple of the warp size");
    __device__ __forceinline__ static void pos(int n_i, int *x) {
        if (D == 2) {
            x[0] = n_i / S1;
            x[1] = n_i % S1;
        } else {
            x[0] = n_i / (S1 * S2);
            x[1] = (n_i / S2) % S1;
            x[2] = n_i % S2;
        }
    }
    __device__ __forceinline__ static int extent(int k) { return k == 0 ? S0 : (k == 1 ? S1 : S2); }
    __device__ __forceinline__ static int local(const int *y) {
        return D == 2 ? y[0] * S1 + y[1] : (y[0] * S1 + y[1]) * S2 + y[2];
    }
};

// Per-instance geometry helpers (shape: true grid shape, shape_o: tiles per axis).
template <int D, class TL>
__device__ __forceinline__ int bilevel_index(const int *y, const int *shape_o) {
    int n_o = 0, n_i = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int s = TL::extent(k);
        const int yo = y[k] / s, yi = y[k] - yo * s;
        n_o = n_o * shape_o[k] + yo;
        n_i = n_i * s + yi;
    }
    return n_o * TL::SIZE + n_i;
}

// ---------------------------------------------------------------- Selling ---
// <x, m y> for integer vectors x, y and m packed lower-triangular.  Follows the
// accumulation order of the reference's scal_vmv (cuda/Geometry_.h).
template <int D>
__device__ __forceinline__ float scal_vmv(const int *x, const float *m, const int *y) {
    float r = 0.f;
    int k = 0;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j, ++k)
            r += float(i == j ? x[i] * y[i] : x[i] * y[j] + x[j] * y[i]) * m[k];
    return r;
}

// Selling's algorithm: obtuse superbase by cyclic reduction from the canonical
// superbase, then weights -<b_i, m b_j> and offsets perp(b_k)
// (agd/Eikonal/HFM_CUDA/cuda/Geometry2.h:21-48).  The cyclic loop is unrolled by
// its period so that every superbase index is a compile-time constant.
__device__ __forceinline__ void selling2(const float *m, float *w, int (*e)[3]) {
    int b0[2] = {1, 0}, b1[2] = {0, 1}, b2[2] = {-1, -1};
    int iter = 0, red = 0;
#define AGD_SELL2_STEP(BI, BJ, BK)                                   \
    if (iter >= 100 || red >= 3) goto done;                          \
    if (scal_vmv<2>(BI, m, BJ) > 0.f) {                              \
        BK[0] = BI[0] - BJ[0]; BK[1] = BI[1] - BJ[1];                 \
        BI[0] = -BI[0]; BI[1] = -BI[1];                              \
        red = 0;                                                     \
    }                                                                \
    ++iter; ++red;
    while (true) {
        AGD_SELL2_STEP(b0, b1, b2)
        AGD_SELL2_STEP(b1, b2, b0)
        AGD_SELL2_STEP(b2, b0, b1)
    }
#undef AGD_SELL2_STEP
done:
    w[0] = fmaxf(0.f, -scal_vmv<2>(b0, m, b1)); e[0][0] = -b2[1]; e[0][1] = b2[0];
    w[1] = fmaxf(0.f, -scal_vmv<2>(b1, m, b2)); e[1][0] = -b0[1]; e[1][1] = b0[0];
    w[2] = fmaxf(0.f, -scal_vmv<2>(b2, m, b0)); e[2][0] = -b1[1]; e[2][1] = b1[0];
}

__device__ __forceinline__ void cross3(const int *a, const int *b, int *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// 3D: the reduction visits the six pairs {i,j} of the superbase cyclically, in
// the order (01)(02)(03)(12)(13)(23); a positive <b_i, m b_j> is fixed by
// b_k += b_i, b_l += b_i, b_i = -b_i.  Offsets are b_k x b_l
// (agd/Eikonal/HFM_CUDA/cuda/Geometry3.h:22-58).
__device__ __forceinline__ void selling3(const float *m, float *w, int (*e)[3]) {
    int b0[3] = {1, 0, 0}, b1[3] = {0, 1, 0}, b2[3] = {0, 0, 1}, b3[3] = {-1, -1, -1};
    int iter = 0, red = 0;
#define AGD_SELL3_STEP(BI, BJ, BK, BL)                               \
    if (iter >= 100 || red >= 6) goto done;                          \
    if (scal_vmv<3>(BI, m, BJ) > 0.f) {                              \
        _Pragma("unroll") for (int c = 0; c < 3; ++c) {              \
            BK[c] += BI[c]; BL[c] += BI[c]; BI[c] = -BI[c];          \
        }                                                            \
        red = 0;                                                     \
    }                                                                \
    ++iter; ++red;
    while (true) {
        AGD_SELL3_STEP(b0, b1, b2, b3)
        AGD_SELL3_STEP(b0, b2, b1, b3)
        AGD_SELL3_STEP(b0, b3, b1, b2)
        AGD_SELL3_STEP(b1, b2, b0, b3)
        AGD_SELL3_STEP(b1, b3, b0, b2)
        AGD_SELL3_STEP(b2, b3, b0, b1)
    }
#undef AGD_SELL3_STEP
done:
    w[0] = fmaxf(0.f, -scal_vmv<3>(b0, m, b1)); cross3(b2, b3, e[0]);
    w[1] = fmaxf(0.f, -scal_vmv<3>(b0, m, b2)); cross3(b1, b3, e[1]);
    w[2] = fmaxf(0.f, -scal_vmv<3>(b0, m, b3)); cross3(b1, b2, e[2]);
    w[3] = fmaxf(0.f, -scal_vmv<3>(b1, m, b2)); cross3(b0, b3, e[3]);
    w[4] = fmaxf(0.f, -scal_vmv<3>(b1, m, b3)); cross3(b0, b2, e[4]);
    w[5] = fmaxf(0.f, -scal_vmv<3>(b2, m, b3)); cross3(b0, b1, e[5]);
}

// ------------------------------------------------------ eikonal operator ---
// Sorting network on (value, weight) pairs, ascending values.  A comparator
// keeps its pair only when strictly ordered, which is the tie rule of the
// reference's index networks (cuda/NetworkSort.h:17-60), so equal values end
// in the same relative order.
__device__ __forceinline__ void cswap(float *v, float *w, int i, int j) {
    const bool keep = v[i] < v[j];
    const float vi = v[i], vj = v[j], wi = w[i], wj = w[j];
    v[i] = keep ? vi : vj; v[j] = keep ? vj : vi;
    w[i] = keep ? wi : wj; w[j] = keep ? wj : wi;
}
template <int N>
__device__ __forceinline__ void sort_pairs(float *v, float *w) {
    if (N == 2) {
        cswap(v, w, 0, 1);
    } else if (N == 3) {
        cswap(v, w, 1, 2); cswap(v, w, 0, 2); cswap(v, w, 0, 1);
    } else if (N == 6) {
        cswap(v, w, 1, 2); cswap(v, w, 4, 5);
        cswap(v, w, 0, 2); cswap(v, w, 3, 5);
        cswap(v, w, 0, 1); cswap(v, w, 3, 4); cswap(v, w, 2, 5);
        cswap(v, w, 0, 3); cswap(v, w, 1, 4);
        cswap(v, w, 2, 4); cswap(v, w, 1, 3);
        cswap(v, w, 2, 3);
    }
}

// Solves sum_k w_k (u - v_k)_+^2 = rhs^2 for u by accumulating the sorted
// neighbour values until the root lies in the current interval
// (agd/Eikonal/HFM_CUDA/cuda/HFM.h:142-190).  v and w are clobbered (sorted).
template <int NACT>
__device__ __forceinline__ float hfm_update(float rhs, float *v, float *w) {
    sort_pairs<NACT>(v, w);
    const float vmin = v[0];
    if (vmin == finf()) return vmin;
    float a = w[0], b = 0.f, c = -rhs * rhs;
    bool stop = false;
#pragma unroll
    for (int q = 1; q < NACT; ++q) {
        const float t = v[q] - vmin;
        stop = stop || ((a * t - 2.f * b) * t + c > 0.f);
        if (!stop) {
            a += w[q];
            b += w[q] * t;
            c += w[q] * t * t;
        }
    }
    const float delta = b * b - a * c;
    // Approximate square root and quotient (a few ulp): the result is compared
    // with tolerances of ~5e-6 relative, and the hardware forms save ~15
    // instructions per update over the correctly rounded ones.
    float sd;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(sd) : "f"(fmaxf(0.f, delta)));
    const float value = a == 0.f ? finf() : __fdividef(b + sd, a);
    return vmin + value;
}

// ---------------------------------------------------- source factorisation ---
// At a point x (relative to the seed) the neighbour values at x - e and x + e
// are shifted by f0 = |x| - |x-e| - <e, m x>/|x| and f1 = |x| - |x+e| +
// <e, m x>/|x| (norms of the seed's metric m): the scheme is then exact for the
// distance to the seed (cuda/EuclideanFactor.h:8-26).  The differences of norms
// are formed as quotients, without cancellation.  xx = <x,mx>, xe = <x,me>, ee = <e,me>.
__device__ __forceinline__ void factor_pair(float xx, float xe, float ee, float &f0, float &f1) {
    const float nx = sqrtf(xx), nm = sqrtf(xx - 2.f * xe + ee), np = sqrtf(xx + 2.f * xe + ee);
    const float g = xe / nx;
    f0 = (2.f * xe - ee) / (nx + nm) - g;
    f1 = (-2.f * xe - ee) / (nx + np) + g;
}

// <x, m y> for the factorisation metric: packed lower triangle (Riemann) or diagonal.
template <int D, bool DIAG>
__device__ __forceinline__ float factor_dot(const float *m, const float *x, const float *y) {
    float r = 0.f;
    if (DIAG) {
#pragma unroll
        for (int i = 0; i < D; ++i) r += m[i] * x[i] * y[i];
        return r;
    }
    int k = 0;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j, ++k) r += (i == j ? x[i] * y[i] : x[i] * y[j] + x[j] * y[i]) * m[k];
    return r;
}

// Second order scheme: the shifts g0, g1 of the neighbours x - 2e and x + 2e,
// g0 = 2 f0 - ((|x| - |x-e|) + (|x-2e| - |x-e|)) and likewise on the other
// side (the second differences of the norm |x| - 2|x-e| + |x-2e| added to the
// first order shift; cuda/EuclideanFactor.h:20-28), each difference of norms
// again a quotient.
__device__ __forceinline__ void factor_pair2(float xx, float xe, float ee, float f0, float f1, float &g0,
                                             float &g1) {
    const float nx = sqrtf(xx), nm = sqrtf(xx - 2.f * xe + ee), np = sqrtf(xx + 2.f * xe + ee);
    const float nm2 = sqrtf(xx - 4.f * xe + 4.f * ee), np2 = sqrtf(xx + 4.f * xe + 4.f * ee);
    const float d0 = (2.f * xe - ee) / (nx + nm), d1 = (-2.f * xe - ee) / (nx + np);  // |x| - |x-/+e|
    const float e0 = (-2.f * xe + 3.f * ee) / (nm + nm2), e1 = (2.f * xe + 3.f * ee) / (np + np2);  // |x-/+2e| - |x-/+e|
    g0 = 2.f * f0 - (d0 + e0);
    g1 = 2.f * f1 - (d1 + e1);
}

// Shifts f[2k], f[2k+1] of the neighbours x -/+ e_k of grid point xt (0 outside
// the radius); with f2, those of x -/+ 2 e_k for the second order scheme.
template <int D, int NACT, bool DIAG>
__device__ __forceinline__ void factor_shifts(const agd_instance &A, const int *xt, const int (*e)[3], float *f,
                                              float *f2 = nullptr) {
    float xr[3] = {0.f, 0.f, 0.f}, r2 = 0.f;
#pragma unroll
    for (int c = 0; c < D; ++c) {
        xr[c] = float(xt[c]) - A.factor_origin[c];
        r2 += xr[c] * xr[c];
    }
    const bool in = r2 < A.factor_radius2;
    const float xx = factor_dot<D, DIAG>(A.factor_metric, xr, xr);
#pragma unroll
    for (int k = 0; k < NACT; ++k) {
        float ek[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int c = 0; c < D; ++c) ek[c] = float(e[k][c]);
        float f0 = 0.f, f1 = 0.f, g0 = 0.f, g1 = 0.f;
        if (in) {
            const float xe = factor_dot<D, DIAG>(A.factor_metric, xr, ek), ee = factor_dot<D, DIAG>(A.factor_metric, ek, ek);
            factor_pair(xx, xe, ee, f0, f1);
            if (f2) factor_pair2(xx, xe, ee, f0, f1, g0, g1);
        }
        f[2 * k] = f0;
        f[2 * k + 1] = f1;
        if (f2) {
            f2[2 * k] = g0;
            f2[2 * k + 1] = g1;
        }
    }
}

// ------------------------------------------------------------------ walls ---
// n / d rounded to the closest integer, halves away from zero (the rounding of
// the reference's divRoundClosest, cuda/Walls.h:12-14).
__device__ __forceinline__ int div_round_closest(int n, int d) {
    return ((n < 0) != (d < 0)) ? (n - d / 2) / d : (n + d / 2) / d;
}

// Whether the segment from grid point xt to xt + v meets no wall
// (cuda/Walls.h:18-50).  wd0 is the wall distance at xt; dist(y) gives the
// wall distance at grid point y (255 outside the grid).  Clear when xt is far
// from every wall (255) or |v|_1 < wd0; otherwise the lattice points
// w_k = round(k v / |v|_inf), k = 1..|v|_inf, are walked from the source: the
// segment is clear as soon as |v - w_k|_1 is below the wall distance at
// xt + w_k, and blocked when xt + w_k is a wall.
template <int D, class Dist>
__device__ __forceinline__ bool visible(int wd0, const int *xt, const int *v, Dist &&dist) {
    if (wd0 == 255) return true;
    int l1 = 0, linf = 0;
#pragma unroll
    for (int c = 0; c < D; ++c) {
        l1 += abs(v[c]);
        linf = max(linf, abs(v[c]));
    }
    if (l1 < wd0) return true;
    for (int k = 1; k <= linf; ++k) {
        int y[3] = {0, 0, 0}, rest = 0;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const int w = div_round_closest(v[c] * k, linf);
            rest += abs(v[c] - w);
            y[c] = xt[c] + w;
        }
        const int d = dist(y);
        if (rest < d) return true;
        if (d == 0) return false;
    }
    return true;
}

// ----------------------------------------------------------- grid barrier ---
// Software grid barrier for cooperatively launched kernels.  Waits are bounded
// in time (globaltimer); a timeout raises AGD_STATUS_WATCHDOG in *err and the
// caller must leave.  Returns false if an error is pending.
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ inline bool grid_barrier(GridBarrier *bar, unsigned int nblocks, unsigned int *err,
                                    unsigned long long timeout_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned int g = ld_acquire(&bar->gen);
        __threadfence();
        if (atomicAdd(&bar->count, 1u) == nblocks - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            const unsigned long long t0 = globaltimer();
            while (ld_acquire(&bar->gen) == g) {
                if (ld_acquire(err) != 0u) { ok = 0; break; }
                if (globaltimer() - t0 > timeout_ns) {
                    atomicOr(err, (unsigned)AGD_STATUS_WATCHDOG);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        if (ld_acquire(err) != 0u) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace agd
