// Persistent, device-scheduled block-iterative eikonal solver for B200
// (Isotropic2/3, Riemann2/3), plus the flow pass and the layout kernels.
//
// Scheduling.  The reference iterates on the host: every outer iteration it
// compacts the flags of the tiles to update (cp.flatnonzero), tests for
// termination (np.any, a device->host sync) and launches `Update` on the
// active tiles (agd/Eikonal/HFM_CUDA/_solvers.py:94-120).  Here one launch of
// resident worker warps runs all outer iterations ("epochs") of all the
// instances of a plan, with no grid-wide barrier: tiles wait in one global
// device queue as (tile, epoch) entries; a visit appends the tiles to revisit
// at the next epoch to its instance's next list (deduplicated by an
// epoch-stamped flag), and the warp that finishes the last tile of an
// instance's epoch publishes that instance's next list to the queue.  Each
// instance therefore follows the reference's epoch semantics exactly (the
// fast-iterative-method scores of cuda/Propagation.h:103-167 are
// epoch-stamped, per instance), while instances never wait for one another.
//
// Tile visit.  One warp per tile (points n_i = lane + 32 p), tile values in
// shared memory, niter_i local sweeps with __syncwarp between phases, and an
// early exit when a full sweep changes nothing (the state is then a fixed point
// of the visit, so the result equals that of the remaining sweeps).  Values of
// neighbours outside the tile are read once per visit through L2 (ld.cg), as
// other SMs update them concurrently.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "sched.cuh"

namespace agd {

// ------------------------------------------------------- stencil cache ---
// Offsets of the Selling stencil packed in one 32-bit word: two 15-bit signed
// fields in 2D, three 10-bit signed fields in 3D; bits 30 and 31 flag the
// neighbours x - e and x + e hidden by a wall (kHideShift).
constexpr int kHideShift = 30;
template <int D>
__device__ __forceinline__ bool pack_offset(const int *e, int &word) {
    if constexpr (D == 2) {
        if (e[0] < -16384 || e[0] > 16383 || e[1] < -16384 || e[1] > 16383) return false;
        word = (e[0] & 0x7fff) | ((e[1] & 0x7fff) << 15);
        return true;
    } else {
        for (int c = 0; c < 3; ++c)
            if (e[c] < -512 || e[c] > 511) return false;
        word = (e[0] & 0x3ff) | ((e[1] & 0x3ff) << 10) | ((e[2] & 0x3ff) << 20);
        return true;
    }
}
template <int D>
__device__ __forceinline__ void unpack_offset(int word, int *e) {
    if (D == 2) {
        e[0] = (word << 17) >> 17;
        e[1] = (word << 2) >> 17;
    } else {
        e[0] = (word << 22) >> 22;
        e[1] = (word << 12) >> 22;
        e[2] = (word << 2) >> 22;
    }
}

// Bilevel index of grid point y of instance I (tile shape at run time).
__device__ __forceinline__ long long bilevel_index_rt(const Inst &I, int D, const int *y) {
    long long n_o = 0, n_i = 0;
    for (int k = 0; k < D; ++k) {
        const int s = I.a.shape_i[k], yo = y[k] / s;
        n_o = n_o * I.shape_o[k] + yo;
        n_i = n_i * s + (y[k] - yo * s);
    }
    return n_o * I.size_i + n_i;
}

// Wall distance at grid point y (255 outside the grid, as at padding).
template <int D, class Index>
__device__ __forceinline__ int wall_dist_at(const agd_instance &A, const int *y, Index &&index) {
    bool in = true;
#pragma unroll
    for (int c = 0; c < D; ++c) in = in && y[c] >= 0 && y[c] < A.shape[c];
    return in ? (int)__ldg(A.wall_dist + index(y)) : 255;
}

// Hidden-neighbour bits (bit s: the neighbour x + (2s - 1) e) of offset e at
// grid point xt, wd0 the wall distance there (cuda/Walls.h:18-50 for both signs).
template <int D, class Index>
__device__ __forceinline__ unsigned hidden_bits(const agd_instance &A, int wd0, const int *xt, const int *e,
                                                Index &&index) {
    if (wd0 == 255) return 0u;
    unsigned h = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        int v[3] = {0, 0, 0};
#pragma unroll
        for (int c = 0; c < D; ++c) v[c] = (2 * s - 1) * e[c];
        if (!visible<D>(wd0, xt, v, [&](const int *y) { return wall_dist_at<D>(A, y, index); })) h |= 1u << s;
    }
    return h;
}

// Instance of global tile t (binary search over the tile bases).
__device__ __forceinline__ const Inst &inst_of_tile(const Inst *insts, int ninst, int t) {
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (insts[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    return insts[lo];
}

// Selling stencil of every point of the Riemann instances of a launch, once per
// solve (the reference recomputes it at each visit, cuda/Riemann_.h:23-29).
// One warp per tile.
template <int D>
__global__ void stencil_kernel(const Inst *insts, int ninst, int total_tiles, Ctrl *ctrl) {
    constexpr int SD = D * (D + 1) / 2;
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= total_tiles) return;
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (insts[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    const Inst &I = insts[lo];
    if (!I.stencil) return;
    const long long base = (long long)(t - I.tile_base) * I.size_i;
    const float *__restrict__ geom = I.a.geom;
    float *__restrict__ out = I.stencil;
    // two points of the lane per step, their loads issued together
    for (int n0 = lane; n0 < I.size_i; n0 += 64) {
        float m[2][SD];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int c = 0; c < SD; ++c)
                m[q][c] = n0 + 32 * q < I.size_i ? __ldg(geom + (size_t)c * I.size_tot + base + n0 + 32 * q) : 1.f;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (n0 + 32 * q >= I.size_i) break;
            const long long n_t = base + n0 + 32 * q;
            float w[SD];
            int e[SD][3];
            if (D == 2) selling2(m[q], w, e);
            else selling3(m[q], w, e);
#pragma unroll
            for (int r = 0; r < SD; ++r) {
                int word = 0;
                if (!pack_offset<D>(e[r], word)) atomicOr(&ctrl->err, (unsigned)AGD_STATUS_UNSUPPORTED);
                __stcs(out + (size_t)r * I.size_tot + n_t, w[r]);
                __stcs(out + (size_t)(SD + r) * I.size_tot + n_t, __int_as_float(word));
            }
        }
    }
}

// Wall visibility of the cached stencils (cuda/FiniteDifferences.h:51-59): for
// the Riemann instances with walls, the hidden-neighbour bits of every offset,
// set in its packed word.  Only points within the wall distance bound walk
// their offsets (Walls.h:18-50).  One warp per tile, after stencil_kernel.
template <int D>
__global__ void stencil_walls_kernel(const Inst *insts, int ninst, int total_tiles) {
    constexpr int SD = D * (D + 1) / 2;
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= total_tiles) return;
    const Inst &I = inst_of_tile(insts, ninst, t);
    if (!I.stencil || !I.a.wall_dist) return;
    const int n_o = t - I.tile_base;
    const long long base = (long long)n_o * I.size_i;
    for (int n_i = lane; n_i < I.size_i; n_i += 32) {
        const long long n_t = base + n_i;
        const int wd0 = __ldg(I.a.wall_dist + n_t);  // 255 far from the walls and at padding
        if (wd0 == 255) continue;
        int xt[3] = {0, 0, 0}, ro = n_o, ri = n_i;
        for (int k = D - 1; k >= 0; --k) {
            xt[k] = (ro % I.shape_o[k]) * I.a.shape_i[k] + ri % I.a.shape_i[k];
            ro /= I.shape_o[k];
            ri /= I.a.shape_i[k];
        }
        for (int r = 0; r < SD; ++r) {
            float *slot = I.stencil + (size_t)(SD + r) * I.size_tot + n_t;
            const int word = __float_as_int(*slot);
            int e[3] = {0, 0, 0};
            unpack_offset<D>(word, e);
            const unsigned h = hidden_bits<D>(I.a, wd0, xt, e, [&](const int *y) { return bilevel_index_rt(I, D, y); });
            if (h) *slot = __int_as_float(word | (int)(h << kHideShift));
        }
    }
}

// Multiprecision buffers, one warp per tile.  dir 0: first -> second buffers
// (before the solve); dir 1: second -> first buffers for the instances whose
// last epoch was odd (after the solve).
__global__ void mp_copy_kernel(Sched S, int dir) {
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= 0 && S.ninst > 0) {
        int lo = 0, hi = S.ninst - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (S.inst[mid].tile_base <= t) lo = mid; else hi = mid - 1;
        }
        const Inst &I = S.inst[lo];
        if (t >= I.tile_base + I.size_o || I.a.multip_step == 0.f) return;
        if (dir == 1 && (S.stats[lo].niter_o & 1) == 0) return;
        const long long base = (long long)(t - I.tile_base) * I.size_i;
        float *uf = dir == 0 ? I.a.values : I.a.values_next, *ut = dir == 0 ? I.a.values_next : I.a.values;
        int *qf = dir == 0 ? I.a.valuesq : I.a.valuesq_next, *qt = dir == 0 ? I.a.valuesq_next : I.a.valuesq;
        for (int n_i = lane; n_i < I.size_i; n_i += 32) {
            ut[base + n_i] = uf[base + n_i];
            qt[base + n_i] = qf[base + n_i];
        }
    }
}

// ------------------------------------------------------------- tile visit ---
// MP: multiprecision, u + uq * multip_step with uq an int32 (cuda/HFM.h:12-25):
// Jacobi sweeps inside the tile and double-buffered epochs, as the reference
// forces strict_iter_i and strict_iter_o with it (_Kernel.py:39-45).
// FACT: source factorisation (shifted neighbour values near the seed).
// MODEL Rander: the Riemann stencil of the first symdim geometry planes, and
// the neighbour values at x -/+ e shifted by +/-<w, e> for the drift w of the
// next ndim planes (FiniteDifferences.h:41-45).
// ORD2: second order scheme (neighbours two steps away, cuda/HFM.h:91-138).
// WALLS: neighbours hidden by a wall read +inf (bits of the stencil cache).
template <class TL, int MODEL, bool MP = false, bool FACT = false, bool ORD2 = false, bool WALLS = false>
struct Visit {
    static constexpr int D = TL::D, P = TL::P;
    static constexpr bool kSelling = MODEL == AGD_MODEL_RIEMANN || MODEL == AGD_MODEL_RANDER;
    static constexpr bool kDrift = MODEL == AGD_MODEL_RANDER;
    static constexpr bool SHIFT = FACT || kDrift;  // neighbour values shifted (fsh)
    static constexpr int NACT = kSelling ? D * (D + 1) / 2 : D;
    static constexpr int NTOT = 2 * NACT;
    static constexpr int SD = D * (D + 1) / 2;

    static constexpr int kBoxed = (int)0xffc00000;  // negative quiet NaN: an in-tile index follows
    // Multiprecision comparison and normalisation (cuda/HFM.h:12-25).
    __device__ __forceinline__ static bool greater(float u, int uq, float v, int vq, float step) {
        return u - v > (float)(vq - uq) * step;
    }
    __device__ __forceinline__ static void normalize(float &u, int &uq, float umax, float step) {
        if (u < umax) {
            const int n = (int)(u / step);
            u -= (float)n * step;
            uq += n;
        }
    }
    __device__ __forceinline__ static void neighbour_mp(float x, int xq, const float *us, const int *uqs, float &v,
                                                        int &vq) {
        const int b = __float_as_int(x);
        const bool in = (b >> 22) == -1;
        const int li = b & (TL::SIZE - 1);
        v = in ? us[li] : x;
        vq = in ? uqs[li] : xq;
    }
    // Shared memory of a warp: the tile's values, then (64-point tiles without
    // multiprecision) one slot per lane and stencil neighbour for the values
    // read from outside the tile, so that every neighbour of a sweep is one
    // shared load; otherwise (kSlots false) the integer parts with multiprecision.
    static constexpr bool kSlots = !MP && TL::SIZE <= 64;
    // Point p of a lane: the 8x8 tiles in two checkerboard colours (p = 0 the
    // points with x0 + x1 even), so that a local sweep updates one colour from
    // the other's values of the same sweep and information crosses the tile in
    // fewer sweeps (batch 128 of Riemann2 512^2: +1.7 %, one instance: +5 %,
    // against rows 0-3 then rows 4-7); the 16x16 tiles in bands of four rows
    // (p >> 1), each in the two colours (p & 1), except at second order
    // (Isotropic2 256^2: 3.68 -> 2.97 ms per solve, 38 -> 30 epochs, against
    // bands of two rows); other tiles lane + 32 p.
    __device__ __forceinline__ static int point_of(int lane, int p) {
        if constexpr (D == 2 && TL::SIZE == 64 && TL::S1 == 8) {
            const int r = lane >> 2;
            return r * 8 + (((lane & 3) << 1) | ((r ^ p) & 1));
        } else if constexpr (D == 2 && TL::SIZE == 256 && TL::S1 == 16 && !ORD2) {
            const int r = 4 * (p >> 1) + (lane >> 3);
            return r * 16 + (((lane & 7) << 1) | ((r ^ p) & 1));
        } else {
            return lane + 32 * p;
        }
    }
    static constexpr int kSmemFloats = kSlots ? TL::SIZE + (ORD2 ? 2 : 1) * P * NTOT * 32 : 2 * TL::SIZE;
    __device__ __forceinline__ static float neighbour(float x, const float *us) {
        const int b = __float_as_int(x);
        const float inside = us[b & (TL::SIZE - 1)];  // index masked into this warp's tile
        return (b >> 22) == -1 ? inside : x;
    }
    // Second order corrections (cuda/HFM.h:91-138): with u0 the point's value and
    // v[k] the smaller neighbour along e_k (on side[k]), where
    // |u0 - 2 v + v2| < thr * max_k (u0 - v_k) and u0 > v, v2 the next neighbour
    // on that side, v becomes v + (v - v2) / 3 and its weight 9/4 of itself.
    // Returns the mask of the corrected neighbours.
    template <class Far>
    __device__ __forceinline__ static unsigned order2(float u0, float *v, float *w, const int *side, Far &&far,
                                                      float thr) {
        float bound = 0.f;
#pragma unroll
        for (int k = 0; k < NACT; ++k) bound = fmaxf(bound, u0 - v[k]);
        unsigned mask = 0;
#pragma unroll
        for (int k = 0; k < NACT; ++k) {
            const float v2 = far(k, side[k]);
            const float d2 = fabsf(u0 - 2.f * v[k] + v2);
            if (d2 < thr * bound && u0 > v[k]) {
                v[k] = (float)((double)v[k] + (double)(v[k] - v2) / 3.0);
                w[k] *= 2.25f;
                mask |= 1u << k;
            }
        }
        return mask;
    }
    __device__ __forceinline__ static float lds(unsigned addr) {
        float v;
        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
        return v;
    }

    // Stencil of the point with bilevel index n_t, in two steps so that the
    // loads of all the points of a lane are in flight together: the raw words
    // (cached weights and packed offsets, or the dual metric; Diagonal: the
    // weights), then the weights and offsets (unpacked, or by Selling's
    // decomposition; unit offsets for Isotropic and Diagonal).
    static constexpr int kRaw = MODEL == AGD_MODEL_ISOTROPIC ? 1 : (MODEL == AGD_MODEL_DIAGONAL ? D : 2 * SD + (kDrift ? D : 0));
    __device__ __forceinline__ static void stencil_load(const Inst &I, size_t n_t, float *raw) {
        if constexpr (MODEL == AGD_MODEL_ISOTROPIC) return;
        if constexpr (MODEL == AGD_MODEL_DIAGONAL) {
#pragma unroll
            for (int k = 0; k < D; ++k) raw[k] = __ldg(I.a.geom + (size_t)k * I.size_tot + n_t);
            return;
        }
        if (I.stencil) {
#pragma unroll
            for (int r = 0; r < 2 * SD; ++r) raw[r] = __ldg(I.stencil + (size_t)r * I.size_tot + n_t);
        } else {
#pragma unroll
            for (int c = 0; c < SD; ++c) raw[c] = __ldg(I.a.geom + (size_t)c * I.size_tot + n_t);
        }
        if constexpr (kDrift) {  // the drift, after the stencil words
#pragma unroll
            for (int c = 0; c < D; ++c) raw[2 * SD + c] = __ldg(I.a.geom + (size_t)(SD + c) * I.size_tot + n_t);
        }
    }
    // Drift shifts <w, e_k> of the offsets (scal_vv order), w = raw[2 SD ..].
    __device__ __forceinline__ static void drift_shifts(const float *raw, const int (*e)[3], float *f) {
#pragma unroll
        for (int k = 0; k < NACT; ++k) {
            float s = 0.f;
#pragma unroll
            for (int c = 0; c < D; ++c) s += raw[2 * SD + c] * float(e[k][c]);
            f[2 * k] += s;
            f[2 * k + 1] -= s;
        }
    }
    // hide[k]: the hidden-neighbour bits of offset k (WALLS: from the cache; else 0).
    // Isotropic offsets are unit vectors, hidden exactly when the neighbour is a
    // wall point, whose value is +inf already: no bits are needed.
    __device__ __forceinline__ static void stencil_decode(const Inst &I, const float *raw, float *w, int (*e)[3],
                                                          unsigned *hide) {
#pragma unroll
        for (int k = 0; k < NACT; ++k) hide[k] = 0u;
        if constexpr (!kSelling) {
#pragma unroll
            for (int k = 0; k < D; ++k) {
                w[k] = MODEL == AGD_MODEL_ISOTROPIC ? I.a.iso_weights[k] : raw[k];
#pragma unroll
                for (int c = 0; c < 3; ++c) e[k][c] = (c == k);
            }
        } else if (I.stencil) {
#pragma unroll
            for (int r = 0; r < SD; ++r) {
                w[r] = raw[r];
                unpack_offset<D>(__float_as_int(raw[SD + r]), e[r]);
                if constexpr (WALLS) hide[r] = (unsigned)__float_as_int(raw[SD + r]) >> kHideShift;
            }
        } else {
            float m[SD];
#pragma unroll
            for (int c = 0; c < SD; ++c) m[c] = raw[c];
            if (D == 2) selling2(m, w, e);
            else selling3(m, w, e);
        }
    }

    __device__ __forceinline__ static void stencil(const Inst &I, size_t n_t, float *w, int (*e)[3]) {
        float raw[kRaw];
        unsigned hide[NACT];
        stencil_load(I, n_t, raw);
        stencil_decode(I, raw, w, e, hide);
    }

    __device__ static void run(const Sched &S, const Inst &I, int ii, int n_o, int e, int lane, float *us) {
        const agd_instance &A = I.a;
        int xo[3] = {0, 0, 0};
        {
            int r = n_o;
#pragma unroll
            for (int k = D - 1; k >= 0; --k) {
                xo[k] = r % I.shape_o[k];
                r /= I.shape_o[k];
            }
        }
        // Scores of this tile and of its neighbours at epoch e-1 (complete): loaded
        // now, so that their latency overlaps the visit (cuda/Propagation.h:103-167).
        const int t = I.tile_base + n_o;
        int nb = -1;  // neighbour tile handled by this lane (lanes 0..2D-1)
        if (lane < 2 * D) {
            int y[3] = {xo[0], xo[1], xo[2]};
            y[lane >> 1] += 2 * (lane & 1) - 1;
            bool ok = true;
#pragma unroll
            for (int k = 0; k < D; ++k) ok = ok && y[k] >= 0 && y[k] < I.shape_o[k];
            if (ok) {
                int m = 0;
#pragma unroll
                for (int k = 0; k < D; ++k) m = m * I.shape_o[k] + y[k];
                nb = I.tile_base + m;
            }
        }
        const int sp_self = (int)score_at(S, t, e - 1);
        const int sp_nb = nb >= 0 ? (int)score_at(S, nb, e - 1) : 0;

        const size_t base = (size_t)n_o * TL::SIZE;
        // Epoch e reads buffer (e-1)&1 and writes buffer e&1 with multiprecision.
        const float *u_in = A.values;
        float *u_out = A.values;
        const int *q_in = nullptr;
        int *q_out = nullptr;
        const float step = A.multip_step;
        if constexpr (MP) {
            const bool odd = (e & 1) != 0;
            u_in = odd ? A.values : A.values_next;
            u_out = odd ? A.values_next : A.values;
            q_in = odd ? A.valuesq : A.valuesq_next;
            q_out = odd ? A.valuesq_next : A.valuesq;
        }
        int *uqs = reinterpret_cast<int *>(us + TL::SIZE);  // integer parts, after the float parts
        float uold[P], rhs[P];
        int qold[P];
        float wts[P][NACT];
        // Neighbour of each stencil offset.  With kSlots: the shared-memory address
        // of its value (the tile slot, or this lane's slot holding the value read
        // from outside).  Otherwise: its value when outside the tile (read once
        // per visit), or its in-tile index boxed as a negative-NaN payload (no
        // solution value is a NaN), so one register holds either.
        float nbv[kSlots ? 1 : P][kSlots ? 1 : NTOT];
        int nbq[MP ? P : 1][MP ? NTOT : 1];
        unsigned nba[kSlots ? P : 1][kSlots ? NTOT : 1];
        float fsh[SHIFT ? P : 1][SHIFT ? NTOT : 1];  // factorisation and drift shifts of the neighbour values
        // second order with factorisation: the shifts of the neighbours two steps away
        float fsh2[FACT && ORD2 ? P : 1][FACT && ORD2 ? NTOT : 1];
        int nbq2[MP && ORD2 ? P : 1][MP && ORD2 ? NTOT : 1];  // their integer parts (multiprecision)
        // second order: the neighbours two steps away, as nba / nbv
        unsigned nba2[ORD2 && kSlots ? P : 1][ORD2 && kSlots ? NTOT : 1];
        float nbv2[ORD2 && !kSlots ? P : 1][ORD2 && !kSlots ? NTOT : 1];
        const unsigned us_addr = (unsigned)__cvta_generic_to_shared(us);
        bool seed[P];
        float raw[P][kRaw];
        // every load of the prologue that does not depend on another one is issued first
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const size_t n_t = base + point_of(lane, p);
            uold[p] = __ldcg(u_in + n_t);
            seed[p] = (__ldg(A.seedbits + (n_t >> 3)) >> (n_t & 7)) & 1;
            rhs[p] = __ldg(A.rhs + n_t);
            if constexpr (MP) qold[p] = __ldcg(q_in + n_t);
            stencil_load(I, n_t, raw[p]);
        }
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int n_i = point_of(lane, p);
            int xi[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
            TL::pos(n_i, xi);
#pragma unroll
            for (int k = 0; k < D; ++k) xt[k] = xo[k] * TL::extent(k) + xi[k];
            if constexpr (MP) {
                float u0 = uold[p];
                int q0 = qold[p];
                if (seed[p]) {
                    u0 = rhs[p];
                    q0 = 0;
                    normalize(u0, q0, A.multip_max, step);
                }
                us[n_i] = u0;
                uqs[n_i] = q0;
            } else {
                us[n_i] = seed[p] ? rhs[p] : uold[p];
            }
            int ev[NACT][3];
            unsigned hide[NACT];
            if (seed[p]) continue;  // seeds (and padding) keep their value: no stencil needed
            stencil_decode(I, raw[p], wts[p], ev, hide);
            if constexpr (SHIFT) {
                if constexpr (FACT) {
                    if constexpr (ORD2) factor_shifts<D, NACT, !kSelling>(A, xt, ev, fsh[p], fsh2[p]);
                    else factor_shifts<D, NACT, !kSelling>(A, xt, ev, fsh[p]);
                } else {
#pragma unroll
                    for (int k = 0; k < NTOT; ++k) fsh[p][k] = 0.f;
                }
                if constexpr (kDrift) drift_shifts(raw[p], ev, fsh[p]);
            }
#pragma unroll
            for (int k = 0; k < NACT; ++k) {
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int eps = 2 * s - 1;
                    // a neighbour hidden by a wall reads +inf, and so does the one after it
                    // (cuda/FiniteDifferences.h:53-59)
                    const bool hidden = WALLS && ((hide[k] >> s) & 1u);
                    int yi[3] = {0, 0, 0}, yt[3] = {0, 0, 0};
                    bool intile = !hidden, indom = !hidden;
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        const int off = eps * ev[k][c];
                        yi[c] = xi[c] + off;
                        yt[c] = xt[c] + off;
                        intile = intile && yi[c] >= 0 && yi[c] < TL::extent(c);
                        indom = indom && yt[c] >= 0 && yt[c] < A.shape[c];
                    }
                    if constexpr (!kSlots) {
                        if (intile) {
                            nbv[p][2 * k + s] = __int_as_float(kBoxed | TL::local(yi));
                        } else {
                            const int ny = indom ? bilevel_index<D, TL>(yt, I.shape_o) : 0;
                            nbv[p][2 * k + s] = indom ? __ldcg(u_in + ny) : finf();
                            if constexpr (MP) nbq[p][2 * k + s] = indom ? __ldcg(q_in + ny) : 0;
                        }
                    } else {
                        int slot = TL::local(yi);
                        if (!intile) {
                            slot = TL::SIZE + (p * NTOT + 2 * k + s) * 32 + lane;
                            const int ny = indom ? bilevel_index<D, TL>(yt, I.shape_o) : 0;
                            us[slot] = indom ? __ldcg(u_in + ny) : finf();
                        }
                        nba[p][2 * k + s] = us_addr + 4u * (unsigned)slot;
                    }
                    if constexpr (ORD2) {  // the neighbour x + 2 eps e_k
                        bool in2 = !hidden, dom2 = !hidden;
#pragma unroll
                        for (int c = 0; c < D; ++c) {
                            const int off = 2 * eps * ev[k][c];
                            yi[c] = xi[c] + off;
                            yt[c] = xt[c] + off;
                            in2 = in2 && yi[c] >= 0 && yi[c] < TL::extent(c);
                            dom2 = dom2 && yt[c] >= 0 && yt[c] < A.shape[c];
                        }
                        if constexpr (kSlots) {
                            int slot = TL::local(yi);
                            if (!in2) {
                                slot = TL::SIZE + P * NTOT * 32 + (p * NTOT + 2 * k + s) * 32 + lane;
                                us[slot] = dom2 ? __ldcg(u_in + bilevel_index<D, TL>(yt, I.shape_o)) : finf();
                            }
                            nba2[p][2 * k + s] = us_addr + 4u * (unsigned)slot;
                        } else {
                            const int ny2 = dom2 ? bilevel_index<D, TL>(yt, I.shape_o) : 0;
                            float v2o = dom2 ? __ldcg(u_in + ny2) : finf();
                            if constexpr (FACT) v2o += fsh2[p][2 * k + s];  // outside the tile: value + shift
                            nbv2[p][2 * k + s] = in2 ? __int_as_float(kBoxed | TL::local(yi)) : v2o;
                            if constexpr (MP) nbq2[p][2 * k + s] = (!in2 && dom2) ? __ldcg(q_in + ny2) : 0;
                        }
                    }
                }
            }
        }
        __syncwarp();
        for (int it = 0; it < A.niter_i; ++it) {
            bool moved = false;
            if constexpr (MP) {
                // strict sweeps: every point from the state at the start of the sweep
                float cand[P];
                int candq[P];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    cand[p] = finf();
                    candq[p] = 0;
                    if (seed[p]) continue;
                    float v[NACT], w[NACT];
                    int vq[NACT];
                    int side[ORD2 ? NACT : 1];
#pragma unroll
                    for (int k = 0; k < NACT; ++k) {
                        float a, b;
                        int aq, bq;
                        neighbour_mp(nbv[p][2 * k], nbq[p][2 * k], us, uqs, a, aq);
                        neighbour_mp(nbv[p][2 * k + 1], nbq[p][2 * k + 1], us, uqs, b, bq);
                        if constexpr (SHIFT) {  // the float part carries the shift (HFM.h:46-53)
                            a += fsh[p][2 * k];
                            b += fsh[p][2 * k + 1];
                        }
                        const bool take_b = greater(a, aq, b, bq, step);  // HFM.h:52-57
                        v[k] = take_b ? b : a;
                        vq[k] = take_b ? bq : aq;
                        w[k] = wts[p][k];
                        if constexpr (ORD2) side[k] = take_b;
                    }
                    int vqmin = kIntMax;  // HFM.h:79-87
#pragma unroll
                    for (int k = 0; k < NACT; ++k)
                        if (v[k] < finf()) vqmin = min(vqmin, vq[k]);
#pragma unroll
                    for (int k = 0; k < NACT; ++k) v[k] += (float)(vq[k] - vqmin) * step;
                    if constexpr (ORD2) {
                        // second order with multiprecision (HFM.h:89-135): the point's value and
                        // the farther neighbours' relative to the integer part vqmin; a farther
                        // neighbour inside the tile takes its factorisation shift after that,
                        // one outside carries it in its float part already
                        const int n_i = point_of(lane, p);
                        if (vqmin != kIntMax) {
                            const float u0 = us[n_i] + (float)(uqs[n_i] - vqmin) * step;
                            order2(u0, v, w, side, [&](int k, int sd) {
                                const float x = nbv2[p][2 * k + sd];
                                const int b = __float_as_int(x);
                                if ((b >> 22) == -1) {
                                    const int li = b & (TL::SIZE - 1);
                                    float r = us[li] + (float)(uqs[li] - vqmin) * step;
                                    if constexpr (FACT) r += fsh2[p][2 * k + sd];
                                    return r;
                                }
                                return x + (float)(nbq2[p][2 * k + sd] - vqmin) * step;
                            }, A.order2_threshold);
                        }
                    }
                    float c = hfm_update<NACT>(rhs[p], v, w);
                    int cq = vqmin;
                    if (c == finf()) cq = 0;
                    else normalize(c, cq, A.multip_max, step);
                    cand[p] = c;
                    candq[p] = cq;
                }
                __syncwarp();
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const int n_i = point_of(lane, p);
                    if (!seed[p] && greater(us[n_i], uqs[n_i], cand[p], candq[p], step)) {
                        us[n_i] = cand[p];
                        uqs[n_i] = candq[p];
                        moved = true;
                    }
                }
                __syncwarp();
            } else {
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const int n_i = point_of(lane, p);
                    float cand = finf();
                    if (!seed[p]) {
                        float v[NACT], w[NACT];
                        int side[ORD2 ? NACT : 1];
#pragma unroll
                        for (int k = 0; k < NACT; ++k) {
                            float a, b;
                            if constexpr (kSlots) {
                                a = lds(nba[p][2 * k]);
                                b = lds(nba[p][2 * k + 1]);
                            } else {
                                a = neighbour(nbv[p][2 * k], us);
                                b = neighbour(nbv[p][2 * k + 1], us);
                            }
                            if constexpr (SHIFT) {
                                a += fsh[p][2 * k];
                                b += fsh[p][2 * k + 1];
                            }
                            if constexpr (ORD2) v[k] = a > b ? b : a;
                            else v[k] = fminf(a, b);  // (no value is a NaN; one instruction)
                            w[k] = wts[p][k];
                            if constexpr (ORD2) side[k] = a > b;
                        }
                        if constexpr (ORD2) order2(us[n_i], v, w, side, [&](int k, int sd) {
                            // (with factorisation, the shift of x +/- 2 e_k; outside the tile
                            // without slots nbv2 carries it already)
                            if constexpr (kSlots) {
                                float r = lds(nba2[p][2 * k + sd]);
                                if constexpr (FACT) r += fsh2[p][2 * k + sd];
                                return r;
                            } else {
                                const float x = nbv2[p][2 * k + sd];
                                if ((__float_as_int(x) >> 22) != -1) return x;
                                float r = us[__float_as_int(x) & (TL::SIZE - 1)];
                                if constexpr (FACT) r += fsh2[p][2 * k + sd];
                                return r;
                            }
                        }, A.order2_threshold);
                        cand = hfm_update<NACT>(rhs[p], v, w);
                    }
                    __syncwarp();
                    if (!seed[p] && us[n_i] > cand) {
                        us[n_i] = cand;
                        moved = true;
                    }
                    __syncwarp();
                }
            }
            if (!__any_sync(kFull, moved)) break;
        }
        bool notconv = false;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int n_i = point_of(lane, p);
            const float u = us[n_i];
            __stcg(u_out + base + n_i, u);
            float diff, uabs;
            if constexpr (MP) {
                const int q = uqs[n_i];
                __stcg(q_out + base + n_i, q);
                diff = fabsf(uold[p] - u + (float)(qold[p] - q) * step);  // Update.h:212-216
                uabs = fabsf(u + (float)q * step);
            } else {
                diff = fabsf(uold[p] - u);
                uabs = fabsf(u);
            }
            const float tol = A.atol + A.rtol * uabs;
            if (!(isnan(diff) || diff <= tol)) notconv = true;
        }
        const bool changed = __any_sync(kFull, notconv);
        __syncwarp();

        // Adaptive Gauss-Seidel iteration: a changed tile is visited again with
        // its neighbours (cuda/Propagation.h:151-154, Neighbor() including the
        // tile itself); global iteration: every tile at every epoch until an
        // epoch changes nothing (_solvers.py:77-92, stop test in close_epoch).
        if (A.flags & (AGD_FLAG_SOLVER_AGSI | AGD_FLAG_SOLVER_GLOBAL)) {
            if (A.flags & AGD_FLAG_SOLVER_GLOBAL) {
                if (changed && lane == 0) atomicMax(&S.ist[ii].changed, e);
                if (lane == 2 * D) push_tile(S, I, ii, t, e);
            } else {
                const int target = !changed ? -1 : lane == 2 * D ? t : nb;
                if (target >= 0) push_tile(S, I, ii, target, e);
            }
            return;
        }
        // Fast iterative method (cuda/Propagation.h:103-167).
        const int front = A.fim_front_width;
        int sn;
        bool prop;
        if (!changed) {
            const int sp = sp_self;
            if (sp == 0 || sp == front) { sn = 0; prop = false; }
            else { sn = front; prop = true; }
        } else {
            sn = 1;
            if (front > 2) {
                const int sq = nb >= 0 ? sp_nb - 1 : -1;
                int mx = sq;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
                sn = max(sn, mx);
            }
            prop = sn > 1;
        }
        if (lane == 0) {
            unsigned *arr = (e & 1) ? S.score1 : S.score0;
            __stcg(arr + t, ((unsigned)e << 8) | (unsigned)sn);
        }
        // The pushes of the tile itself (lane 2D, when changed) and of its
        // neighbours (lanes 0..2D-1) go out together.
        const int target = lane == 2 * D ? (changed ? t : -1) : (prop ? nb : -1);
        if (target >= 0) push_tile(S, I, ii, target, e);
    }
};

template <unsigned long long VMASK>
__device__ __forceinline__ void dispatch(const Sched &S, int t, int ii, int e, int lane, float *us) {
    const Inst &I = S.inst[ii];
    const int n_o = t - I.tile_base;
    switch (I.variant) {
        case V_ISO2_8:
            if constexpr ((VMASK >> V_ISO2_8) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_ISOTROPIC>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_16:
            if constexpr ((VMASK >> V_ISO2_16) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8:
            if constexpr ((VMASK >> V_RIEM2_8) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO3_4:
            if constexpr ((VMASK >> V_ISO3_4) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4:
            if constexpr ((VMASK >> V_RIEM3_4) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_16:
            if constexpr ((VMASK >> V_RIEM2_16) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_RIEMANN>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_8_MP:
            if constexpr ((VMASK >> V_ISO2_8_MP) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_ISOTROPIC, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_16_MP:
            if constexpr ((VMASK >> V_ISO2_16_MP) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8_MP:
            if constexpr ((VMASK >> V_RIEM2_8_MP) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, true, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO3_4_MP:
            if constexpr ((VMASK >> V_ISO3_4_MP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4_MP:
            if constexpr ((VMASK >> V_RIEM3_4_MP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, true, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_8_F:
            if constexpr ((VMASK >> V_ISO2_8_F) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_ISOTROPIC, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_16_FMP:
            if constexpr ((VMASK >> V_ISO2_16_FMP) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8_FMP:
            if constexpr ((VMASK >> V_RIEM2_8_FMP) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, true, true, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO3_4_FMP:
            if constexpr ((VMASK >> V_ISO3_4_FMP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4_FMP:
            if constexpr ((VMASK >> V_RIEM3_4_FMP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, true, true, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_16_O2F:
            if constexpr ((VMASK >> V_ISO2_16_O2F) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, false, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8_O2F:
            if constexpr ((VMASK >> V_RIEM2_8_O2F) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, false, true, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO3_4_O2F:
            if constexpr ((VMASK >> V_ISO3_4_O2F) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, false, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4_O2F:
            if constexpr ((VMASK >> V_RIEM3_4_O2F) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, false, true, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_16_O2MP:
            if constexpr ((VMASK >> V_ISO2_16_O2MP) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, true, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8_O2MP:
            if constexpr ((VMASK >> V_RIEM2_8_O2MP) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, true, false, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO3_4_O2MP:
            if constexpr ((VMASK >> V_ISO3_4_O2MP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, true, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4_O2MP:
            if constexpr ((VMASK >> V_RIEM3_4_O2MP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, true, false, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_16_O2FMP:
            if constexpr ((VMASK >> V_ISO2_16_O2FMP) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, true, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8_O2FMP:
            if constexpr ((VMASK >> V_RIEM2_8_O2FMP) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, true, true, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO3_4_O2FMP:
            if constexpr ((VMASK >> V_ISO3_4_O2FMP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, true, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4_O2FMP:
            if constexpr ((VMASK >> V_RIEM3_4_O2FMP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, true, true, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_16_F:
            if constexpr ((VMASK >> V_ISO2_16_F) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8_F:
            if constexpr ((VMASK >> V_RIEM2_8_F) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, false, true, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO3_4_F:
            if constexpr ((VMASK >> V_ISO3_4_F) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4_F:
            if constexpr ((VMASK >> V_RIEM3_4_F) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, false, true, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_8_O2:
            if constexpr ((VMASK >> V_ISO2_8_O2) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_ISOTROPIC, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO2_16_O2:
            if constexpr ((VMASK >> V_ISO2_16_O2) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8_O2:
            if constexpr ((VMASK >> V_RIEM2_8_O2) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, false, false, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_ISO3_4_O2:
            if constexpr ((VMASK >> V_ISO3_4_O2) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4_O2:
            if constexpr ((VMASK >> V_RIEM3_4_O2) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, false, false, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_8_W:
            if constexpr ((VMASK >> V_RIEM2_8_W) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, false, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM2_16_W:
            if constexpr ((VMASK >> V_RIEM2_16_W) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_RIEMANN, false, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RIEM3_4_W:
            if constexpr ((VMASK >> V_RIEM3_4_W) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, false, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG2_8:
            if constexpr ((VMASK >> V_DIAG2_8) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_DIAGONAL>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG2_16:
            if constexpr ((VMASK >> V_DIAG2_16) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_DIAGONAL>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG3_4:
            if constexpr ((VMASK >> V_DIAG3_4) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_DIAGONAL>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG2_8_MP:
            if constexpr ((VMASK >> V_DIAG2_8_MP) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_DIAGONAL, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG2_16_MP:
            if constexpr ((VMASK >> V_DIAG2_16_MP) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_DIAGONAL, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG3_4_MP:
            if constexpr ((VMASK >> V_DIAG3_4_MP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_DIAGONAL, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG2_8_F:
            if constexpr ((VMASK >> V_DIAG2_8_F) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_DIAGONAL, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG2_16_F:
            if constexpr ((VMASK >> V_DIAG2_16_F) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_DIAGONAL, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG3_4_F:
            if constexpr ((VMASK >> V_DIAG3_4_F) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_DIAGONAL, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG2_8_O2:
            if constexpr ((VMASK >> V_DIAG2_8_O2) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_DIAGONAL, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG2_16_O2:
            if constexpr ((VMASK >> V_DIAG2_16_O2) & 1) Visit<Tile<2, 16, 16, 1>, AGD_MODEL_DIAGONAL, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_DIAG3_4_O2:
            if constexpr ((VMASK >> V_DIAG3_4_O2) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_DIAGONAL, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND2_8:
            if constexpr ((VMASK >> V_RAND2_8) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND3_4:
            if constexpr ((VMASK >> V_RAND3_4) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND2_8_W:
            if constexpr ((VMASK >> V_RAND2_8_W) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER, false, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND3_4_W:
            if constexpr ((VMASK >> V_RAND3_4_W) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER, false, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND2_8_MP:
            if constexpr ((VMASK >> V_RAND2_8_MP) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER, true, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND3_4_MP:
            if constexpr ((VMASK >> V_RAND3_4_MP) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER, true, false, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND2_8_F:
            if constexpr ((VMASK >> V_RAND2_8_F) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER, false, true, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND3_4_F:
            if constexpr ((VMASK >> V_RAND3_4_F) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER, false, true, false, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND2_8_O2:
            if constexpr ((VMASK >> V_RAND2_8_O2) & 1) Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER, false, false, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        case V_RAND3_4_O2:
            if constexpr ((VMASK >> V_RAND3_4_O2) & 1) Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER, false, false, true, true>::run(S, I, ii, n_o, e, lane, us);
            break;
        default:
            break;
    }
}

constexpr int kMaxTileSize = 256;

// Shared floats per warp for the variants of VMASK.
template <unsigned long long VMASK>
constexpr int smem_floats() {
    int m = 0;
    if ((VMASK >> V_ISO2_8) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_ISOTROPIC>::kSmemFloats);
    if ((VMASK >> V_ISO2_16) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC>::kSmemFloats);
    if ((VMASK >> V_RIEM2_8) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN>::kSmemFloats);
    if ((VMASK >> V_ISO3_4) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC>::kSmemFloats);
    if ((VMASK >> V_RIEM3_4) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN>::kSmemFloats);
    if ((VMASK >> V_RIEM2_16) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_RIEMANN>::kSmemFloats);
    if (VMASK & kMpVariants) m = std::max(m, 2 * kMaxTileSize);
    if ((VMASK >> V_ISO2_8_F) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_ISOTROPIC, false, true>::kSmemFloats);
    if ((VMASK >> V_ISO2_16_F) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, false, true>::kSmemFloats);
    if ((VMASK >> V_RIEM2_8_F) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, false, true, false, true>::kSmemFloats);
    if ((VMASK >> V_ISO3_4_F) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, false, true>::kSmemFloats);
    if ((VMASK >> V_RIEM3_4_F) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, false, true, false, true>::kSmemFloats);
    if ((VMASK >> V_ISO2_8_O2) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_ISOTROPIC, false, false, true>::kSmemFloats);
    if ((VMASK >> V_ISO2_16_O2) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, false, false, true>::kSmemFloats);
    if ((VMASK >> V_RIEM2_8_O2) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, false, false, true, true>::kSmemFloats);
    if ((VMASK >> V_ISO3_4_O2) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, false, false, true>::kSmemFloats);
    if ((VMASK >> V_RIEM3_4_O2) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, false, false, true, true>::kSmemFloats);
    if ((VMASK >> V_RIEM2_8_W) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, false, false, false, true>::kSmemFloats);
    if ((VMASK >> V_RIEM2_16_W) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_RIEMANN, false, false, false, true>::kSmemFloats);
    if ((VMASK >> V_RIEM3_4_W) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, false, false, false, true>::kSmemFloats);
    if ((VMASK >> V_DIAG2_8) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_DIAGONAL>::kSmemFloats);
    if ((VMASK >> V_DIAG2_16) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_DIAGONAL>::kSmemFloats);
    if ((VMASK >> V_DIAG3_4) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_DIAGONAL>::kSmemFloats);
    if ((VMASK >> V_DIAG2_8_F) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_DIAGONAL, false, true>::kSmemFloats);
    if ((VMASK >> V_DIAG2_16_F) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_DIAGONAL, false, true>::kSmemFloats);
    if ((VMASK >> V_DIAG3_4_F) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_DIAGONAL, false, true>::kSmemFloats);
    if ((VMASK >> V_DIAG2_8_O2) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_DIAGONAL, false, false, true>::kSmemFloats);
    if ((VMASK >> V_DIAG2_16_O2) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_DIAGONAL, false, false, true>::kSmemFloats);
    if ((VMASK >> V_DIAG3_4_O2) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_DIAGONAL, false, false, true>::kSmemFloats);
    if ((VMASK >> V_RAND2_8) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER>::kSmemFloats);
    if ((VMASK >> V_RAND3_4) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER>::kSmemFloats);
    if ((VMASK >> V_RAND2_8_W) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER, false, false, false, true>::kSmemFloats);
    if ((VMASK >> V_RAND3_4_W) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER, false, false, false, true>::kSmemFloats);
    if ((VMASK >> V_RAND2_8_F) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER, false, true, false, true>::kSmemFloats);
    if ((VMASK >> V_RAND3_4_F) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER, false, true, false, true>::kSmemFloats);
    if ((VMASK >> V_RAND2_8_O2) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER, false, false, true, true>::kSmemFloats);
    if ((VMASK >> V_RAND3_4_O2) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER, false, false, true, true>::kSmemFloats);
    if ((VMASK >> V_ISO2_16_O2F) & 1) m = std::max(m, Visit<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC, false, true, true>::kSmemFloats);
    if ((VMASK >> V_RIEM2_8_O2F) & 1) m = std::max(m, Visit<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN, false, true, true, true>::kSmemFloats);
    if ((VMASK >> V_ISO3_4_O2F) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC, false, true, true>::kSmemFloats);
    if ((VMASK >> V_RIEM3_4_O2F) & 1) m = std::max(m, Visit<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN, false, true, true, true>::kSmemFloats);
    return m;
}

template <unsigned long long VMASK, bool BULK = false>
struct EikonalVisitor {
    // Resident 4-warp CTAs per SM the register budget must allow: 256-point tiles
    // keep 8 points per lane in registers, Riemann3 twelve neighbours per point,
    // multiprecision an integer part beside every value.
    // Riemann3 / Rander3: 5 CTAs at up to 96 registers (a single 200^3 solve:
    // 24.1 ms, against 26.1 ms at 6 CTAs and 80 registers with 2.5x the
    // spills, and 29.6 ms at 7).  Riemann2 8x8: 8 CTAs at up to 64 registers
    // (48 bytes of spills; batch 128 of 512^2: +1 % over 9 CTAs at 56 registers
    // and 96 bytes, +7 % over 10 CTAs at 48 registers and 160 bytes).
    // BULK: epochs published in batches (enqueue_warp<true>).  Its registers
    // make the variants at their budget spill (Riemann2 8x8: 164 -> 504 bytes,
    // -13 % solves/s at a batch of 128 instances), but an instance of tens of
    // thousands of tiles per epoch is bound by its publication (Riemann3 200^3:
    // -13 % solve time, Riemann2 1024^2: -5 %): plans of a few large instances
    // use these instantiations (run_variants).
    static constexpr bool kBulkPublish = BULK;
    // (the BULK instantiations serve plans of fewer than kPairInstances instances)
    static constexpr bool kBatchScheduling = !BULK;
    static constexpr int kMinCtas =
        (VMASK & ((1ull << V_RIEM2_16) | (1ull << V_ISO2_16) | (1ull << V_ISO2_16_MP) | (1ull << V_ISO2_16_F) |
                  (1ull << V_ISO2_16_FMP) | (1ull << V_ISO2_16_O2F) | (1ull << V_ISO2_16_O2MP) |
                  (1ull << V_ISO2_16_O2FMP) |
                  (1ull << V_ISO2_16_O2) | (1ull << V_RIEM2_16_W) | (1ull << V_DIAG2_16) |
                  (1ull << V_DIAG2_16_MP) | (1ull << V_DIAG2_16_F) | (1ull << V_DIAG2_16_O2)))      ? 4
        : (VMASK & ((1ull << V_RIEM3_4) | (1ull << V_RIEM3_4_MP) | (1ull << V_RIEM3_4_F) | (1ull << V_RIEM3_4_O2) |
                    (1ull << V_RIEM3_4_W) | (1ull << V_RAND3_4) | (1ull << V_RAND3_4_W) | (1ull << V_RAND3_4_MP) |
                    (1ull << V_RAND3_4_F) | (1ull << V_RAND3_4_O2) | (1ull << V_RIEM3_4_FMP) |
                    (1ull << V_RIEM3_4_O2F) | (1ull << V_RIEM3_4_O2MP) | (1ull << V_RIEM3_4_O2FMP))) ? 5
        : (VMASK & (kMpVariants | kFactorVariants | kOrder2Variants))                                ? 7
        : (VMASK & (1ull << V_RIEM2_8))                                                              ? 8
                                                                                                     : 9;
    struct Args {};
    struct Smem {
        float u[smem_floats<VMASK>()];  // values, then out-of-tile neighbours or integer parts
    };
    __device__ __forceinline__ static void visit(const Sched &S, const Args &, int t, int ii, int e, int lane, Smem &sm) {
        dispatch<VMASK>(S, t, ii, e, lane, sm.u);
    }
    // Before the workers: the second buffers of multiprecision instances start
    // as copies of the first (_SetArgs.py:171-177), and the Selling stencils of
    // the Riemann instances are computed.
    static cudaError_t prepare(const Sched &S, const WsLayout &L, cudaStream_t st) {
        constexpr unsigned long long kRiemann = (1ull << V_RIEM2_8) | (1ull << V_RIEM3_4) | (1ull << V_RIEM2_16) |
                                      (1ull << V_RIEM2_8_MP) | (1ull << V_RIEM3_4_MP) | (1ull << V_RIEM2_8_F) |
                                      (1ull << V_RIEM3_4_F) | (1ull << V_RIEM2_8_O2) | (1ull << V_RIEM3_4_O2) |
                                      (1ull << V_RIEM2_8_FMP) | (1ull << V_RIEM3_4_FMP) | kWallVariants |
                                      kRanderVariants | (1ull << V_RIEM2_8_O2F) | (1ull << V_RIEM3_4_O2F) |
                                      (1ull << V_RIEM2_8_O2MP) | (1ull << V_RIEM3_4_O2MP) |
                                      (1ull << V_RIEM2_8_O2FMP) | (1ull << V_RIEM3_4_O2FMP);
        if (VMASK & kMpVariants) mp_copy_kernel<<<(L.total_tiles + 7) / 8, 256, 0, st>>>(S, 0);
        if (!(VMASK & kRiemann) || L.stencil == L.total) return cudaGetLastError();
        // variants that read the hidden-neighbour bits: the walls pass follows
        constexpr unsigned long long kWallCapable = kWallVariants | (1ull << V_RIEM2_8_MP) | (1ull << V_RIEM3_4_MP) |
                                          (1ull << V_RIEM2_8_F) | (1ull << V_RIEM3_4_F) | (1ull << V_RIEM2_8_O2) |
                                          (1ull << V_RIEM3_4_O2) | (1ull << V_RIEM2_8_FMP) | (1ull << V_RIEM3_4_FMP) |
                                          (1ull << V_RIEM2_8_O2F) | (1ull << V_RIEM3_4_O2F) | (1ull << V_RIEM2_8_O2MP) |
                                          (1ull << V_RIEM3_4_O2MP) | (1ull << V_RIEM2_8_O2FMP) | (1ull << V_RIEM3_4_O2FMP) |
                                          (kRanderVariants & ~((1ull << V_RAND2_8) | (1ull << V_RAND3_4)));
        const unsigned grid = (L.total_tiles + 7) / 8;
        if (VMASK & ((1ull << V_RIEM3_4) | (1ull << V_RIEM3_4_MP) | (1ull << V_RIEM3_4_F) | (1ull << V_RIEM3_4_O2) |
                     (1ull << V_RIEM3_4_W) | (1ull << V_RAND3_4) | (1ull << V_RAND3_4_W) | (1ull << V_RAND3_4_MP) |
                     (1ull << V_RAND3_4_F) | (1ull << V_RAND3_4_O2) | (1ull << V_RIEM3_4_FMP) |
                     (1ull << V_RIEM3_4_O2F) | (1ull << V_RIEM3_4_O2MP) | (1ull << V_RIEM3_4_O2FMP))) {
            stencil_kernel<3><<<grid, 256, 0, st>>>(S.inst, S.ninst, L.total_tiles, S.ctrl);
            if (VMASK & kWallCapable) stencil_walls_kernel<3><<<grid, 256, 0, st>>>(S.inst, S.ninst, L.total_tiles);
        } else {
            stencil_kernel<2><<<grid, 256, 0, st>>>(S.inst, S.ninst, L.total_tiles, S.ctrl);
            if (VMASK & kWallCapable) stencil_walls_kernel<2><<<grid, 256, 0, st>>>(S.inst, S.ninst, L.total_tiles);
        }
        return cudaGetLastError();
    }
    // After the workers: an instance that ran an odd number of epochs has its
    // result in the second buffers (the reference swaps its argument names).
    static cudaError_t finalize(const Sched &S, const WsLayout &L, cudaStream_t st) {
        if (VMASK & kMpVariants) mp_copy_kernel<<<(L.total_tiles + 7) / 8, 256, 0, st>>>(S, 1);
        return cudaGetLastError();
    }
};

}  // namespace agd

struct agd_plan {
    std::vector<agd::Inst> insts;
    agd::WsLayout L;
    unsigned long long vmask;
    int ndim;
};

namespace agd {

// Checks the instances of one launch; returns the mask of tile-visit variants.
// stencil_cache: whether the launch computes the Riemann stencil cache.
static int validate(const agd_instance *host, const Inst *insts, int n, bool stencil_cache, unsigned long long *vmask) {
    *vmask = 0;
    for (int i = 0; i < n; ++i) {
        const agd_instance &a = host[i];
        const char *bad = nullptr;
        int code = AGD_STATUS_INVALID;
        if (a.ndim != host[0].ndim) bad = "all instances of a plan must share ndim";
        else if (insts[i].variant < 0) { bad = "model/tile shape not built"; code = AGD_STATUS_UNSUPPORTED; }
        else if (a.wall_dist && (a.model == AGD_MODEL_RIEMANN || a.model == AGD_MODEL_RANDER) && !stencil_cache) {
            bad = "walls on a Riemann instance need the stencil cache (agd_eikonal_solve)";
            code = AGD_STATUS_UNSUPPORTED;
        }
        else if (a.multip_step != 0.f && (!a.valuesq || !a.values_next || !a.valuesq_next || !(a.multip_step > 0.f)))
            bad = "multiprecision needs valuesq, values_next, valuesq_next and multip_step > 0";
        else if (!a.values || !a.rhs || !a.seedbits || (a.model != AGD_MODEL_ISOTROPIC && !a.geom)) bad = "missing array";
        else if (reinterpret_cast<uintptr_t>(a.seedbits) % 4 != 0) bad = "seedbits must be 4-byte aligned";
        else if (a.niter_i < 1 || a.fim_front_width < 2 || a.fim_front_width > 255 || a.nitermax_o < 0 ||
                 a.nitermax_o > kMaxEpochs)
            bad = "bad niter_i / fim_front_width / nitermax_o (at most 16000)";
        if (bad) return set_error(code, bad);
        *vmask |= 1ull << insts[i].variant;
    }
    return AGD_STATUS_OK;
}

static int plan_create(const agd_instance *host, int n, agd_plan **out) {
    if (!out) return set_error(AGD_STATUS_INVALID, "null plan pointer");
    *out = nullptr;
    if (n <= 0 || !host) return set_error(AGD_STATUS_INVALID, "no instance");
    agd_plan *P = new agd_plan();
    if (!layout(host, n, P->L, &P->insts)) {
        delete P;
        return set_error(AGD_STATUS_INVALID, "bad instance shape");
    }
    P->ndim = host[0].ndim;
    const int rc = validate(host, P->insts.data(), n, /*stencil_cache=*/true, &P->vmask);
    if (rc != AGD_STATUS_OK) {
        delete P;
        return rc;
    }
    *out = P;
    return AGD_STATUS_OK;
}

// The persistent solve for the variants in vmask, on a workspace laid out by L
// whose descriptors are already uploaded.
static int run_variants(int ndim, unsigned long long vmask, const WsLayout &L, void *ws, int n, agd_stats *stats,
                        const agd_launch *cfg, cudaStream_t st) {
    constexpr unsigned long long R2 = 1ull << V_RIEM2_8, I16 = 1ull << V_ISO2_16, I8 = 1ull << V_ISO2_8;
    constexpr unsigned long long R3 = 1ull << V_RIEM3_4, I3 = 1ull << V_ISO3_4, R2L = 1ull << V_RIEM2_16;
    constexpr unsigned long long MP2 = (1ull << V_ISO2_8_MP) | (1ull << V_ISO2_16_MP) | (1ull << V_RIEM2_8_MP) |
                                       (1ull << V_ISO2_16_FMP) | (1ull << V_RIEM2_8_FMP);
    constexpr unsigned long long MP3 = (1ull << V_ISO3_4_MP) | (1ull << V_RIEM3_4_MP) | (1ull << V_ISO3_4_FMP) |
                                       (1ull << V_RIEM3_4_FMP);
    // Riemann with walls, beside plain instances of every family
    constexpr unsigned long long W2 = (1ull << V_RIEM2_8_W) | (1ull << V_RIEM2_16_W), W3 = 1ull << V_RIEM3_4_W;
    if (vmask & kRanderVariants) {  // Rander instances run in kernels of their own
        constexpr unsigned long long RB2 = (1ull << V_RAND2_8) | (1ull << V_RAND2_8_W);
        constexpr unsigned long long RB3 = (1ull << V_RAND3_4) | (1ull << V_RAND3_4_W);
        if (vmask & ~kRanderVariants) return set_error(AGD_STATUS_UNSUPPORTED, "Rander instances beside other models in one plan");
        const bool mp = vmask & kMpVariants, f = vmask & kFactorVariants, o2 = vmask & kOrder2Variants;
        if (int(mp) + int(f) + int(o2) > 1)
            return set_error(AGD_STATUS_UNSUPPORTED, "Rander instances of several option families in one plan");
        if (ndim == 2) {
            if (o2) return run_sched<EikonalVisitor<(1ull << V_RAND2_8_O2) | RB2>>(L, ws, n, {}, stats, cfg, st);
            if (f) return run_sched<EikonalVisitor<(1ull << V_RAND2_8_F) | RB2>>(L, ws, n, {}, stats, cfg, st);
            if (mp) return run_sched<EikonalVisitor<(1ull << V_RAND2_8_MP) | RB2>>(L, ws, n, {}, stats, cfg, st);
            return run_sched<EikonalVisitor<RB2>>(L, ws, n, {}, stats, cfg, st);
        }
        if (o2) return run_sched<EikonalVisitor<(1ull << V_RAND3_4_O2) | RB3>>(L, ws, n, {}, stats, cfg, st);
        if (f) return run_sched<EikonalVisitor<(1ull << V_RAND3_4_F) | RB3>>(L, ws, n, {}, stats, cfg, st);
        if (mp) return run_sched<EikonalVisitor<(1ull << V_RAND3_4_MP) | RB3>>(L, ws, n, {}, stats, cfg, st);
        return run_sched<EikonalVisitor<RB3>>(L, ws, n, {}, stats, cfg, st);
    }
    if (vmask & kDiagVariants) {  // Diagonal instances run in kernels of their own
        constexpr unsigned long long D2 = (1ull << V_DIAG2_8) | (1ull << V_DIAG2_16), D3 = 1ull << V_DIAG3_4;
        constexpr unsigned long long DMP2 = (1ull << V_DIAG2_8_MP) | (1ull << V_DIAG2_16_MP), DMP3 = 1ull << V_DIAG3_4_MP;
        constexpr unsigned long long DF2 = (1ull << V_DIAG2_8_F) | (1ull << V_DIAG2_16_F), DF3 = 1ull << V_DIAG3_4_F;
        constexpr unsigned long long DO2 = (1ull << V_DIAG2_8_O2) | (1ull << V_DIAG2_16_O2), DO3 = 1ull << V_DIAG3_4_O2;
        if (vmask & ~kDiagVariants) return set_error(AGD_STATUS_UNSUPPORTED, "Diagonal instances beside other models in one plan");
        const bool mp = vmask & kMpVariants, f = vmask & kFactorVariants, o2 = vmask & kOrder2Variants;
        if (int(mp) + int(f) + int(o2) > 1)
            return set_error(AGD_STATUS_UNSUPPORTED, "Diagonal instances of several option families in one plan");
        if (ndim == 2) {
            if (o2) return run_sched<EikonalVisitor<DO2 | D2>>(L, ws, n, {}, stats, cfg, st);
            if (f) return run_sched<EikonalVisitor<DF2 | D2>>(L, ws, n, {}, stats, cfg, st);
            if (mp) return run_sched<EikonalVisitor<DMP2 | D2>>(L, ws, n, {}, stats, cfg, st);
            return run_sched<EikonalVisitor<D2>>(L, ws, n, {}, stats, cfg, st);
        }
        if (o2) return run_sched<EikonalVisitor<DO3 | D3>>(L, ws, n, {}, stats, cfg, st);
        if (f) return run_sched<EikonalVisitor<DF3 | D3>>(L, ws, n, {}, stats, cfg, st);
        if (mp) return run_sched<EikonalVisitor<DMP3 | D3>>(L, ws, n, {}, stats, cfg, st);
        return run_sched<EikonalVisitor<D3>>(L, ws, n, {}, stats, cfg, st);
    }
    constexpr unsigned long long kO2Combined = kOrder2FactorVariants | kOrder2MpVariants | kOrder2FactorMpVariants;
    if (vmask & kO2Combined) {  // second order with factorisation, multiprecision, or both
        const bool f = vmask & kOrder2FactorVariants, mp = vmask & kOrder2MpVariants,
                   fmp = vmask & kOrder2FactorMpVariants;
        if (int(f) + int(mp) + int(fmp) > 1 || (vmask & ~kO2Combined))
            return set_error(AGD_STATUS_UNSUPPORTED,
                             "second order with factorisation or multiprecision beside other instances in one plan");
        constexpr unsigned long long OF2 = (1ull << V_ISO2_16_O2F) | (1ull << V_RIEM2_8_O2F);
        constexpr unsigned long long OF3 = (1ull << V_ISO3_4_O2F) | (1ull << V_RIEM3_4_O2F);
        constexpr unsigned long long OM2 = (1ull << V_ISO2_16_O2MP) | (1ull << V_RIEM2_8_O2MP);
        constexpr unsigned long long OM3 = (1ull << V_ISO3_4_O2MP) | (1ull << V_RIEM3_4_O2MP);
        constexpr unsigned long long OFM2 = (1ull << V_ISO2_16_O2FMP) | (1ull << V_RIEM2_8_O2FMP);
        constexpr unsigned long long OFM3 = (1ull << V_ISO3_4_O2FMP) | (1ull << V_RIEM3_4_O2FMP);
        if (ndim == 2) return f ? run_sched<EikonalVisitor<OF2>>(L, ws, n, {}, stats, cfg, st)
                              : mp ? run_sched<EikonalVisitor<OM2>>(L, ws, n, {}, stats, cfg, st)
                                   : run_sched<EikonalVisitor<OFM2>>(L, ws, n, {}, stats, cfg, st);
        return f ? run_sched<EikonalVisitor<OF3>>(L, ws, n, {}, stats, cfg, st)
               : mp ? run_sched<EikonalVisitor<OM3>>(L, ws, n, {}, stats, cfg, st)
                    : run_sched<EikonalVisitor<OFM3>>(L, ws, n, {}, stats, cfg, st);
    }
    if (vmask & kOrder2Variants) {  // second order instances, possibly beside plain ones
        constexpr unsigned long long O2 = (1ull << V_ISO2_8_O2) | (1ull << V_ISO2_16_O2) | (1ull << V_RIEM2_8_O2);
        constexpr unsigned long long O3 = (1ull << V_ISO3_4_O2) | (1ull << V_RIEM3_4_O2);
        if (vmask & (kMpVariants | kFactorVariants))
            return set_error(AGD_STATUS_UNSUPPORTED, "second order beside multiprecision or factorisation in one plan");
        if (ndim == 2) return run_sched<EikonalVisitor<O2 | R2 | I16 | I8 | R2L | W2>>(L, ws, n, {}, stats, cfg, st);
        return run_sched<EikonalVisitor<O3 | R3 | I3 | W3>>(L, ws, n, {}, stats, cfg, st);
    }
    if (vmask & kFactorVariants) {  // factored instances, possibly beside plain ones
        constexpr unsigned long long F2 = (1ull << V_ISO2_8_F) | (1ull << V_ISO2_16_F) | (1ull << V_RIEM2_8_F);
        constexpr unsigned long long F3 = (1ull << V_ISO3_4_F) | (1ull << V_RIEM3_4_F);
        if (vmask & kMpVariants)
            return set_error(AGD_STATUS_UNSUPPORTED, "factored instances without and with multiprecision in one plan");
        if (ndim == 2) return run_sched<EikonalVisitor<F2 | R2 | I16 | I8 | R2L | W2>>(L, ws, n, {}, stats, cfg, st);
        return run_sched<EikonalVisitor<F3 | R3 | I3 | W3>>(L, ws, n, {}, stats, cfg, st);
    }
    if (vmask & kMpVariants) {
        if (ndim == 2) {
            if (vmask == (1ull << V_RIEM2_8_MP)) return run_sched<EikonalVisitor<(1ull << V_RIEM2_8_MP)>>(L, ws, n, {}, stats, cfg, st);
            return run_sched<EikonalVisitor<R2 | I16 | I8 | R2L | MP2 | W2>>(L, ws, n, {}, stats, cfg, st);
        }
        return run_sched<EikonalVisitor<R3 | I3 | MP3 | W3>>(L, ws, n, {}, stats, cfg, st);
    }
    // A plan of a few instances of 8192 tiles or more on average: batched epoch
    // publication, for the base variants.
    const bool bulk = n < kPairInstances && (long long)L.total_tiles >= 8192LL * n;
    if (bulk) {
        if (vmask == R2) return run_sched<EikonalVisitor<R2, true>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == R2L) return run_sched<EikonalVisitor<R2L, true>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == I16) return run_sched<EikonalVisitor<I16, true>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == I8) return run_sched<EikonalVisitor<I8, true>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == R3) return run_sched<EikonalVisitor<R3, true>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == I3) return run_sched<EikonalVisitor<I3, true>>(L, ws, n, {}, stats, cfg, st);
    }
    if (ndim == 2) {
        if (vmask == R2) return run_sched<EikonalVisitor<R2>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == R2L) return run_sched<EikonalVisitor<R2L>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == I16) return run_sched<EikonalVisitor<I16>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == I8) return run_sched<EikonalVisitor<I8>>(L, ws, n, {}, stats, cfg, st);
        if (vmask == (1ull << V_RIEM2_8_W)) return run_sched<EikonalVisitor<(1ull << V_RIEM2_8_W)>>(L, ws, n, {}, stats, cfg, st);
        return run_sched<EikonalVisitor<R2 | I16 | I8 | R2L | W2>>(L, ws, n, {}, stats, cfg, st);
    }
    if (vmask == R3) return run_sched<EikonalVisitor<R3>>(L, ws, n, {}, stats, cfg, st);
    if (vmask == I3) return run_sched<EikonalVisitor<I3>>(L, ws, n, {}, stats, cfg, st);
    return run_sched<EikonalVisitor<R3 | I3 | W3>>(L, ws, n, {}, stats, cfg, st);
}

static int plan_run(const agd_plan *P, void *ws, size_t ws_bytes, agd_stats *stats, const agd_launch *cfg,
                    cudaStream_t st) {
    if (!P || !ws) return set_error(AGD_STATUS_INVALID, "null plan or workspace");
    const WsLayout &L = P->L;
    if (ws_bytes < L.total) return set_error(AGD_STATUS_WORKSPACE, "workspace too small");
    return run_variants(P->ndim, P->vmask, L, ws, (int)P->insts.size(), stats, cfg, st);
}

// ------------------------------------------------------- fixed scratch ---
// Scratch of agd_eikonal_solve_fixed_scratch: a file-scope device array, so that
// callers which cannot allocate device memory still get a solver.  In host code
// the name g_fixed_scratch is only a host-side stand-in for the symbol; the
// device address is obtained once per device with cudaGetSymbolAddress.
constexpr size_t kFixedScratchBytes = (size_t)AGD_FIXED_SCRATCH_BYTES;
constexpr int kFixedScratchMaxInstances = AGD_FIXED_SCRATCH_MAX_INSTANCES;
static __device__ __align__(256) unsigned char g_fixed_scratch[kFixedScratchBytes];
constexpr int kMaxDevices = 64;
static void *g_fixed_scratch_addr[kMaxDevices];
static std::mutex g_fixed_scratch_lock;
// Host staging of the instance descriptors (about 64 KiB at the maximum count):
// a file-scope array rather than a stack one, since plugin threads may have
// small stacks.  Used under g_fixed_scratch_lock until the upload has read it.
static Inst g_fixed_scratch_insts[kFixedScratchMaxInstances];

static int fixed_scratch_solve(const agd_instance *host, int n, agd_stats *stats, const agd_launch *cfg,
                               cudaStream_t st) {
    if (!host || n <= 0) return set_error(AGD_STATUS_INVALID, "no instance");
    if (n > kFixedScratchMaxInstances)
        return set_error(AGD_STATUS_INVALID, "agd_eikonal_solve_fixed_scratch: more than "
                                             "AGD_FIXED_SCRATCH_MAX_INSTANCES instances");
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return set_cuda_error("cudaGetDevice", err);
    if (dev < 0 || dev >= kMaxDevices) return set_error(AGD_STATUS_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> guard(g_fixed_scratch_lock);  // held until the descriptors are staged
    if (!g_fixed_scratch_addr[dev]) {  // first call on this device: resolve the array's device address
        err = cudaGetSymbolAddress(&g_fixed_scratch_addr[dev], g_fixed_scratch);
        if (err != cudaSuccess) {
            g_fixed_scratch_addr[dev] = nullptr;
            return set_cuda_error("cudaGetSymbolAddress(fixed scratch)", err);
        }
    }
    void *scratch = g_fixed_scratch_addr[dev];
    Inst *insts = g_fixed_scratch_insts;
    WsLayout L;
    if (!layout(host, n, L, insts, /*stencil_cache=*/false)) return set_error(AGD_STATUS_INVALID, "bad instance shape");
    unsigned long long vmask = 0;
    const int rc = validate(host, insts, n, /*stencil_cache=*/false, &vmask);
    if (rc != AGD_STATUS_OK) return rc;
    if (L.total > kFixedScratchBytes)
        return set_error(AGD_STATUS_WORKSPACE, "agd_eikonal_solve_fixed_scratch: these instances need more "
                                               "scratch than AGD_FIXED_SCRATCH_BYTES; use agd_eikonal_solve");
    // Pageable host source: the call returns once the descriptors are staged,
    // after which the host array may be reused.
    err = cudaMemcpyAsync(static_cast<char *>(scratch) + L.inst, insts, sizeof(Inst) * n, cudaMemcpyHostToDevice, st);
    if (err != cudaSuccess) return set_cuda_error("descriptor upload", err);
    return run_variants(host[0].ndim, vmask, L, scratch, n, stats, cfg, st);
}

static int plan_upload(const agd_plan *P, void *ws, size_t ws_bytes, cudaStream_t st) {
    if (!P || !ws) return set_error(AGD_STATUS_INVALID, "null plan or workspace");
    if (ws_bytes < P->L.total) return set_error(AGD_STATUS_WORKSPACE, "workspace too small");
    std::vector<Inst> insts(P->insts);
    rebase_stencils(insts.data(), (int)insts.size(), P->L, ws);
    // pageable source: the call returns once the descriptors are staged
    const cudaError_t err = cudaMemcpyAsync(static_cast<char *>(ws) + P->L.inst, insts.data(),
                                            sizeof(Inst) * insts.size(), cudaMemcpyHostToDevice, st);
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("descriptor upload", err);
}

// ------------------------------------------------------------------ flow ---
// Upwind flow at every point of a solved instance (FLOW_* exports of
// cuda/Update.h:171-209 with one local iteration).  Values are not modified.
template <class TL, int MODEL>
__global__ void flow_kernel(Inst I, float *fvec, float *fwsum, float *fw, int *fidx) {
    using V = Visit<TL, MODEL>;
    constexpr int D = TL::D, P = TL::P, NACT = V::NACT;
    const int lane = threadIdx.x & 31;
    const int n_o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (n_o >= I.size_o) return;
    const agd_instance &A = I.a;
    int xo[3] = {0, 0, 0};
    {
        int r = n_o;
#pragma unroll
        for (int k = D - 1; k >= 0; --k) { xo[k] = r % I.shape_o[k]; r /= I.shape_o[k]; }
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int n_i = lane + 32 * p;
        const size_t n_t = (size_t)n_o * TL::SIZE + n_i;
        int xi[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
        TL::pos(n_i, xi);
        bool in = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            xt[k] = xo[k] * TL::extent(k) + xi[k];
            in = in && xt[k] < A.shape[k];
        }
        const bool seed = (__ldg(A.seedbits + (n_t >> 3)) >> (n_t & 7)) & 1;
        float w[NACT], fwk[NACT];
        int ev[NACT][3], side[NACT];
        V::stencil(I, n_t, w, ev);
        unsigned hide[NACT];  // neighbours hidden by a wall (Riemann offsets; see Visit::stencil_decode)
        const int wd0 = (V::kSelling && A.wall_dist && in) ? (int)__ldg(A.wall_dist + n_t) : 255;
#pragma unroll
        for (int k = 0; k < NACT; ++k)
            hide[k] = hidden_bits<D>(A, wd0, xt, ev[k], [&](const int *y) { return bilevel_index<D, TL>(y, I.shape_o); });
        float v[NACT], fsh[2 * NACT], fsh2[2 * NACT];
#pragma unroll
        for (int k = 0; k < 2 * NACT; ++k) fsh2[k] = 0.f;
        if (A.factor_radius2 > 0.f) {
            if (A.order2_threshold > 0.f) factor_shifts<D, NACT, !V::kSelling>(A, xt, ev, fsh, fsh2);
            else factor_shifts<D, NACT, !V::kSelling>(A, xt, ev, fsh);
        } else {
#pragma unroll
            for (int k = 0; k < 2 * NACT; ++k) fsh[k] = 0.f;
        }
        if constexpr (V::kDrift) {
            float raw[V::kRaw];
#pragma unroll
            for (int c = 0; c < D; ++c) raw[2 * V::SD + c] = __ldg(A.geom + (size_t)(V::SD + c) * I.size_tot + n_t);
            V::drift_shifts(raw, ev, fsh);
        }
#pragma unroll
        for (int k = 0; k < NACT; ++k) {
            side[k] = 0;
            fwk[k] = 0.f;
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                int y[3] = {0, 0, 0};
                bool ok = !((hide[k] >> s) & 1u);
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    y[c] = xt[c] + (2 * s - 1) * ev[k][c];
                    ok = ok && y[c] >= 0 && y[c] < A.shape[c];
                }
                const float val = (ok ? __ldg(A.values + bilevel_index<D, TL>(y, I.shape_o)) : finf()) + fsh[2 * k + s];
                if (s == 0) v[k] = val;
                else if (v[k] > val) { v[k] = val; side[k] = 1; }
            }
        }
        if (!seed && in) {
            float vs[NACT], ws[NACT];
#pragma unroll
            for (int k = 0; k < NACT; ++k) { vs[k] = v[k]; ws[k] = w[k]; }
            unsigned o2 = 0;
            if (A.order2_threshold > 0.f) {  // second order: v corrected in place, weights 9/4
                o2 = V::order2(__ldg(A.values + n_t), vs, ws, side, [&](int k, int sd) {
                    int y[3] = {0, 0, 0};
                    bool ok = !((hide[k] >> sd) & 1u);
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        y[c] = xt[c] + 2 * (2 * sd - 1) * ev[k][c];
                        ok = ok && y[c] >= 0 && y[c] < A.shape[c];
                    }
                    return (ok ? __ldg(A.values + bilevel_index<D, TL>(y, I.shape_o)) : finf()) + fsh2[2 * k + sd];
                }, A.order2_threshold);
#pragma unroll
                for (int k = 0; k < NACT; ++k) v[k] = vs[k];
            }
            const float val = hfm_update<NACT>(__ldg(A.rhs + n_t), vs, ws);
            if (val != finf()) {
#pragma unroll
                for (int k = 0; k < NACT; ++k)
                    fwk[k] = w[k] * fmaxf(0.f, val - v[k]) * (((o2 >> k) & 1) ? 1.5f : 1.f);
            }
        }
        float vec[3] = {0.f, 0.f, 0.f}, sum = 0.f;
#pragma unroll
        for (int k = 0; k < NACT; ++k) {
            sum += fwk[k];
            const int eps = 2 * side[k] - 1;
            int y[3] = {0, 0, 0};
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const int off = eps * ev[k][c];
                vec[c] += fwk[k] * float(off);
                y[c] = xt[c] + off;
            }
            if (fw) fw[(size_t)k * I.size_tot + n_t] = fwk[k];
            if (fidx) fidx[(size_t)k * I.size_tot + n_t] = fwk[k] != 0.f ? bilevel_index<D, TL>(y, I.shape_o) : kIntMax;
        }
        if (fvec)
#pragma unroll
            for (int c = 0; c < D; ++c) fvec[(size_t)c * I.size_tot + n_t] = vec[c];
        if (fwsum) fwsum[n_t] = sum;
    }
}

static int flow_impl(const agd_instance *a, float *fvec, float *fwsum, float *fw, int *fidx, cudaStream_t st) {
    WsLayout L;
    std::vector<Inst> v;
    if (!a || !layout(a, 1, L, &v, /*stencil_cache=*/false)) return set_error(AGD_STATUS_INVALID, "bad instance");
    const Inst &I = v[0];
    const int wpb = 4, grid = (I.size_o + wpb - 1) / wpb;
    switch (base_variant_of(I.a)) {
        case V_ISO2_8: flow_kernel<Tile<2, 8, 8, 1>, AGD_MODEL_ISOTROPIC><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_ISO2_16: flow_kernel<Tile<2, 16, 16, 1>, AGD_MODEL_ISOTROPIC><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_RIEM2_8: flow_kernel<Tile<2, 8, 8, 1>, AGD_MODEL_RIEMANN><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_ISO3_4: flow_kernel<Tile<3, 4, 4, 4>, AGD_MODEL_ISOTROPIC><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_RIEM3_4: flow_kernel<Tile<3, 4, 4, 4>, AGD_MODEL_RIEMANN><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_RIEM2_16: flow_kernel<Tile<2, 16, 16, 1>, AGD_MODEL_RIEMANN><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_DIAG2_8: flow_kernel<Tile<2, 8, 8, 1>, AGD_MODEL_DIAGONAL><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_DIAG2_16: flow_kernel<Tile<2, 16, 16, 1>, AGD_MODEL_DIAGONAL><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_DIAG3_4: flow_kernel<Tile<3, 4, 4, 4>, AGD_MODEL_DIAGONAL><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_RAND2_8: flow_kernel<Tile<2, 8, 8, 1>, AGD_MODEL_RANDER><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        case V_RAND3_4: flow_kernel<Tile<3, 4, 4, 4>, AGD_MODEL_RANDER><<<grid, wpb * 32, 0, st>>>(I, fvec, fwsum, fw, fidx); break;
        default: return set_error(AGD_STATUS_UNSUPPORTED, "model/tile shape not built");
    }
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("flow_kernel", err);
}

// ---------------------------------------------------------- layout prep ---
struct Geo {
    int nd, shape[3], si[3], so[3], size_i;
    long long size_tot, n;
};
static bool geo_of(int nd, const int *shape, const int *si, Geo &g) {
    if (nd < 1 || nd > 3) return false;
    g.nd = nd;
    g.size_i = 1;
    g.n = 1;
    long long so = 1;
    for (int k = 0; k < 3; ++k) { g.shape[k] = 1; g.si[k] = 1; g.so[k] = 1; }
    for (int k = 0; k < nd; ++k) {
        if (shape[k] <= 0 || si[k] <= 0) return false;
        g.shape[k] = shape[k];
        g.si[k] = si[k];
        g.so[k] = (shape[k] + si[k] - 1) / si[k];
        g.size_i *= si[k];
        so *= g.so[k];
        g.n *= shape[k];
    }
    g.size_tot = so * g.size_i;
    return true;
}

// bilevel index -> grid coordinates (returns false for padding)
__device__ __forceinline__ bool grid_coords(const Geo &g, long long n_t, int *x, long long &flat) {
    long long n_o = n_t / g.size_i;
    int n_i = (int)(n_t - n_o * g.size_i);
    int xo[3], xi[3];
    for (int k = g.nd - 1; k >= 0; --k) {
        xo[k] = (int)(n_o % g.so[k]); n_o /= g.so[k];
        xi[k] = n_i % g.si[k]; n_i /= g.si[k];
    }
    bool in = true;
    flat = 0;
    for (int k = 0; k < g.nd; ++k) {
        x[k] = xo[k] * g.si[k] + xi[k];
        in = in && x[k] < g.shape[k];
        flat = flat * g.shape[k] + x[k];
    }
    return in;
}

__global__ void block_expand_kernel(Geo g, int nplanes, const float *src, int bcast, float pad, float *dst) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.size_tot * nplanes) return;
    const int plane = (int)(i / g.size_tot);
    const long long n_t = i - plane * g.size_tot;
    int x[3];
    long long flat;
    const bool in = grid_coords(g, n_t, x, flat);
    dst[i] = in ? (bcast ? src[plane] : src[plane * g.n + flat]) : pad;
}

__global__ void block_squeeze_kernel(Geo g, int nplanes, const float *src, float *dst) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.n * nplanes) return;
    const int plane = (int)(i / g.n);
    long long r = i - plane * g.n;
    int x[3];
    for (int k = g.nd - 1; k >= 0; --k) { x[k] = (int)(r % g.shape[k]); r /= g.shape[k]; }
    long long n_o = 0, n_i = 0;
    for (int k = 0; k < g.nd; ++k) {
        n_o = n_o * g.so[k] + x[k] / g.si[k];
        n_i = n_i * g.si[k] + x[k] % g.si[k];
    }
    dst[i] = src[plane * g.size_tot + n_o * g.size_i + n_i];
}

// Dual metric of M' = diag(h) M diag(h) (Riemann.with_costs, then dual), by the
// adjugate formula, packed [d00, d10, d11(, d20, d21, d22)]; with is_dual, m
// already holds the dual metric and is only rescaled (dualMetric.with_speeds(h)).
__device__ __forceinline__ void geom_at(int nd, const float *m, int is_dual, const float h[3], float *out) {
    if (nd == 2) {
        float a = m[0], b = m[1], c = m[2];
        if (is_dual) {  // entries / (h_i h_j)
            out[0] = a / (h[0] * h[0]); out[1] = b / (h[1] * h[0]); out[2] = c / (h[1] * h[1]);
            return;
        }
        a = a * (h[0] * h[0]); b = b * (h[1] * h[0]); c = c * (h[1] * h[1]);
        const float det = a * c - b * b;
        out[0] = c / det;
        out[1] = -b / det;
        out[2] = a / det;
        return;
    }
    float s[6];
    int k = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j, ++k) s[k] = is_dual ? m[k] / (h[i] * h[j]) : m[k] * (h[i] * h[j]);
    if (is_dual) {
        for (int c = 0; c < 6; ++c) out[c] = s[c];
        return;
    }
    // symmetric [[a,b,d],[b,c,e],[d,e,f]] with s = [a, b, c, d, e, f]
    const float a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5];
    const float A00 = c * f - e * e, A10 = d * e - b * f, A11 = a * f - d * d;
    const float A20 = b * e - c * d, A21 = b * d - a * e, A22 = a * c - b * b;
    const float det = a * A00 + b * A10 + d * A20;
    out[0] = A00 / det; out[1] = A10 / det; out[2] = A11 / det;
    out[3] = A20 / det; out[4] = A21 / det; out[5] = A22 / det;
}

// Geometry planes in tile layout; +inf at padding points.
__global__ void prep_geom_kernel(Geo g, const float *metric, int bcast, int is_dual, double h0, double h1,
                                 double h2, float *geom) {
    const long long n_t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n_t >= g.size_tot) return;
    const int sd = g.nd * (g.nd + 1) / 2;
    int x[3];
    long long flat;
    const bool in = grid_coords(g, n_t, x, flat);
    if (!in) {
        for (int c = 0; c < sd; ++c) geom[c * g.size_tot + n_t] = finf();
        return;
    }
    const float h[3] = {(float)h0, (float)h1, (float)h2};
    float out[6];
    geom_at(g.nd, bcast ? metric : metric + flat * sd, is_dual, h, out);
    for (int c = 0; c < sd; ++c) geom[c * g.size_tot + n_t] = out[c];
}

// Diagonal model: the squared dual costs 1/(c_k h_k)^2 of metric.with_costs(h)
// (or (d_k / h_k)^2 of dualMetric.with_speeds(h)) per axis, in float as the
// reference forms them (_SetGeometry.py:134-135), +inf at padding.
__device__ __forceinline__ void diag_at(int nd, const float *c, int is_dual, const float h[3], float *out) {
    for (int k = 0; k < nd; ++k) {
        const float v = is_dual ? c[k] * (1.f / h[k]) : 1.f / (c[k] * h[k]);
        out[k] = v * v;
    }
}

__global__ void prep_diag_kernel(Geo g, const float *costs, int bcast, int is_dual, double h0, double h1, double h2,
                                 float *geom) {
    const long long n_t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n_t >= g.size_tot) return;
    int x[3];
    long long flat;
    const bool in = grid_coords(g, n_t, x, flat);
    const float h[3] = {(float)h0, (float)h1, (float)h2};
    float out[3];
    if (in) diag_at(g.nd, bcast ? costs : costs + flat * g.nd, is_dual, h, out);
    for (int k = 0; k < g.nd; ++k) geom[k * g.size_tot + n_t] = in ? out[k] : finf();
}

// Inverse of a packed symmetric matrix [a00, a10, a11(, a20, a21, a22)] by the
// adjugate formula.
__device__ __forceinline__ void sym_inverse(int nd, const float *s, float *out) {
    if (nd == 2) {
        const float det = s[0] * s[2] - s[1] * s[1];
        out[0] = s[2] / det;
        out[1] = -s[1] / det;
        out[2] = s[0] / det;
        return;
    }
    const float a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5];
    const float A00 = c * f - e * e, A10 = d * e - b * f, A11 = a * f - d * d;
    const float A20 = b * e - c * d, A21 = b * d - a * e, A22 = a * c - b * b;
    const float det = a * A00 + b * A10 + d * A20;
    out[0] = A00 / det; out[1] = A10 / det; out[2] = A11 / det;
    out[3] = A20 / det; out[4] = A21 / det; out[5] = A22 / det;
}

// Rander model: (inverse of m * outer(h, h), w * h) per point, +inf at padding
// (Metrics/rander.py:61-68).  With is_dual the input (m_d, w_d) is the dual
// metric: scaled by with_speeds(h), then turned into the metric by
// rander.py:35-39, m = (1 + <w_d, s w_d>) s, w = -s w_d with s = (m_d - w_d w_d^T)^-1,
// so that the inverse of m is (m_d - w_d w_d^T) / (1 + <w_d, s w_d>).
// out: the sd planes of the inverse metric, then the nd of the drift.
__device__ __forceinline__ void rander_at(int nd, const float *src, int is_dual, const float hh[3], float *out) {
    const int sd = nd * (nd + 1) / 2;
    float hs[3];  // the grid scales (metric), or their inverses (with_speeds of a dual metric)
    for (int k = 0; k < nd; ++k) hs[k] = is_dual ? 1.f / hh[k] : hh[k];
    float m[6], w[3], mi[6];
    int q = 0;
    for (int i = 0; i < nd; ++i)
        for (int j = 0; j <= i; ++j, ++q) m[q] = src[q] * (hs[i] * hs[j]);  // m * outer(h, h)
    for (int k = 0; k < nd; ++k) w[k] = src[sd + k] * hs[k];
    if (!is_dual) {
        sym_inverse(nd, m, mi);
    } else {
        float t[6], s_[6], om[3] = {0.f, 0.f, 0.f};
        q = 0;
        for (int i = 0; i < nd; ++i)
            for (int j = 0; j <= i; ++j, ++q) t[q] = m[q] - w[i] * w[j];
        sym_inverse(nd, t, s_);
        for (int i = 0; i < nd; ++i)
            for (int j = 0; j < nd; ++j) om[i] += s_[i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i] * w[j];
        float wo = 0.f;
        for (int i = 0; i < nd; ++i) wo += w[i] * om[i];
        for (int c = 0; c < sd; ++c) mi[c] = t[c] / (1.f + wo);
        for (int k = 0; k < nd; ++k) w[k] = -om[k];
    }
    for (int c = 0; c < sd; ++c) out[c] = mi[c];
    for (int k = 0; k < nd; ++k) out[sd + k] = w[k];
}

__global__ void prep_rander_kernel(Geo g, const float *metric, int bcast, int is_dual, double h0, double h1,
                                   double h2, float *geom) {
    const long long n_t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n_t >= g.size_tot) return;
    const int nd = g.nd, sd = nd * (nd + 1) / 2;
    int x[3];
    long long flat;
    const bool in = grid_coords(g, n_t, x, flat);
    const float hh[3] = {(float)h0, (float)h1, (float)h2};
    float out[9];
    if (in) rander_at(nd, bcast ? metric : metric + flat * (sd + nd), is_dual, hh, out);
    for (int c = 0; c < sd + nd; ++c) geom[c * g.size_tot + n_t] = in ? out[c] : finf();
}

// Seed bits: one 32-bit word (32 points) per thread, padding bits set.
__global__ void seedbits_init_kernel(Geo g, unsigned *bits) {
    const long long wi = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (wi * 32 >= g.size_tot) return;
    unsigned word = 0;
    for (int b = 0; b < 32; ++b) {
        int x[3];
        long long flat;
        if (!grid_coords(g, wi * 32 + b, x, flat)) word |= 1u << b;
    }
    bits[wi] = word;
}

// Seeds in order (a later duplicate overrides an earlier one, as numpy assignment does).
// walls (grid layout, or NULL): a seed on a wall keeps the wall's +inf right-hand
// side, since the reference writes the walls after the seeds.
__device__ void place_seeds(const Geo &g, const int *idx, const float *vals, int n, float *rhs, unsigned *bits,
                            unsigned char *trigger, int *bad, const uint8_t *walls = nullptr) {
    for (int s = 0; s < n; ++s) {
        long long n_o = 0, n_i = 0, flat = 0;
        bool ok = true;
        for (int k = 0; k < g.nd; ++k) {
            const int xk = idx[s * g.nd + k];
            ok = ok && xk >= 0 && xk < g.shape[k];
            n_o = n_o * g.so[k] + (ok ? xk / g.si[k] : 0);
            n_i = n_i * g.si[k] + (ok ? xk % g.si[k] : 0);
            flat = flat * g.shape[k] + (ok ? xk : 0);
        }
        if (!ok) {
            if (bad) *bad = 1;
            continue;
        }
        const long long n_t = n_o * g.size_i + n_i;
        if (rhs && !(walls && walls[flat])) rhs[n_t] = vals ? vals[s] : 0.f;
        if (bits) bits[n_t >> 5] |= 1u << (n_t & 31);
        if (trigger) trigger[n_o] = 1;
    }
}

__global__ void seeds_kernel(Geo g, const int *idx, const float *vals, int n, float *rhs, unsigned *bits,
                             unsigned char *trigger, int *bad) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    place_seeds(g, idx, vals, n, rhs, bits, trigger, bad);
}

struct BatchPrep {
    Geo g;
    int si_log2[3];  // log2 of the tile sides, or -1 (all) if one is not a power of two
    int n, model, is_dual, nseeds;
    int nmet, ngeom;  // metric floats per point, geometry planes
    float h[3];
    const float *metric, *cost, *seed_values;
    const int *seed_index;
    float *geom, *rhs, *values;
    unsigned *bits;
    int *bad;
    const uint8_t *walls;
    long long walls_stride;  // 0: one mask for every instance
    uint8_t *trigger;
    long long size_o;  // tiles of an instance
};

// Bilevel index -> grid coordinates for instances of fewer than 2^31 points,
// in 32-bit arithmetic, the in-tile part by shifts when the tile sides are
// powers of two (si_log2 >= 0).  Returns false for padding.
__device__ __forceinline__ bool grid_coords32(const Geo &g, const int *si_log2, int n_t, int &flat) {
    int n_o, n_i, xo[3], xi[3];
    if (si_log2[0] >= 0) {
        const int lsz = si_log2[0] + si_log2[1] + si_log2[2];
        n_o = n_t >> lsz;
        n_i = n_t & ((1 << lsz) - 1);
        for (int k = g.nd - 1; k >= 0; --k) {
            xi[k] = n_i & ((1 << si_log2[k]) - 1);
            n_i >>= si_log2[k];
        }
    } else {
        n_o = n_t / g.size_i;
        n_i = n_t - n_o * g.size_i;
        for (int k = g.nd - 1; k >= 0; --k) {
            xi[k] = n_i % g.si[k];
            n_i /= g.si[k];
        }
    }
    for (int k = g.nd - 1; k >= 0; --k) {
        const int q = n_o / g.so[k];
        xo[k] = n_o - q * g.so[k];
        n_o = q;
    }
    bool in = true;
    flat = 0;
    for (int k = 0; k < g.nd; ++k) {
        const int x = xo[k] * g.si[k] + xi[k];
        in = in && x < g.shape[k];
        flat = flat * g.shape[k] + x;
    }
    return in;
}

// Grid rows of blocks: blockIdx.y is the instance, the blocks of a row stride
// over its points (warps stay 32-aligned because size_tot is a multiple of 32,
// so each warp's ballot is one bit word).
__global__ void prep_batch_kernel(BatchPrep A) {
    const int inst = blockIdx.y;
    const int size_tot = (int)A.g.size_tot;
    for (int n_t = blockIdx.x * blockDim.x + threadIdx.x; n_t < size_tot; n_t += gridDim.x * blockDim.x) {
        const long long i = (long long)inst * size_tot + n_t;
        int flat;
        const bool in = grid_coords32(A.g, A.si_log2, n_t, flat);
        const bool wall = in && A.walls && A.walls[inst * A.walls_stride + flat];
        A.values[i] = finf();
        A.rhs[i] = in && !wall ? (A.cost ? A.cost[inst * A.g.n + flat] : 1.f) : finf();
        if (A.ngeom) {
            float out[9];
            if (in) {
                const float *m = A.metric + (inst * A.g.n + flat) * A.nmet;
                if (A.model == AGD_MODEL_RIEMANN) geom_at(A.g.nd, m, A.is_dual, A.h, out);
                else if (A.model == AGD_MODEL_DIAGONAL) diag_at(A.g.nd, m, A.is_dual, A.h, out);
                else rander_at(A.g.nd, m, A.is_dual, A.h, out);
            }
            float *geo = A.geom + (long long)inst * A.ngeom * A.g.size_tot + n_t;
            for (int c = 0; c < A.ngeom; ++c) geo[c * A.g.size_tot] = in ? out[c] : finf();
        }
        if (A.trigger && n_t % A.g.size_i == 0) A.trigger[inst * A.size_o + n_t / A.g.size_i] = 0;
        const unsigned pad = __ballot_sync(0xffffffffu, !in || wall);
        if ((threadIdx.x & 31) == 0) A.bits[i >> 5] = pad;
    }
}

__global__ void seeds_batch_kernel(BatchPrep A) {
    const int inst = blockIdx.x * blockDim.x + threadIdx.x;
    if (inst >= A.n) return;
    place_seeds(A.g, A.seed_index + (long long)inst * A.nseeds * A.g.nd,
                A.seed_values ? A.seed_values + (long long)inst * A.nseeds : nullptr, A.nseeds,
                A.rhs + inst * A.g.size_tot, A.bits + inst * (A.g.size_tot / 32),
                A.trigger ? A.trigger + inst * A.size_o : nullptr, A.bad,
                A.walls ? A.walls + inst * A.walls_stride : nullptr);
}

// Wall distances in tile layout (255 at padding); with rhs / bits, the wall
// points become seeds of value +inf (_SetArgs.py:124-126).  One thread per
// point; whole warps leave together (size_tot is a multiple of 32), and the
// wall bits of a warp are one seed-bit word, which only that warp writes.
__global__ void walls_kernel(Geo g, const uint8_t *walls, const uint8_t *dist, uint8_t *wall_dist, float *rhs,
                             unsigned *bits) {
    const long long n_t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n_t >= g.size_tot) return;
    int x[3];
    long long flat;
    const bool in = grid_coords(g, n_t, x, flat);
    const bool wall = in && walls[flat] != 0;
    wall_dist[n_t] = in ? dist[flat] : (uint8_t)255;
    if (wall && rhs) rhs[n_t] = finf();
    const unsigned word = __ballot_sync(kFull, wall);
    if (bits && word && (threadIdx.x & 31) == 0) bits[n_t >> 5] |= word;
}

// Wall distances of nb instances, grid layout (dist) -> tile layout (255 at padding).
__global__ void wall_dist_batch_kernel(Geo g, int nb, const uint8_t *dist, uint8_t *wall_dist) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.size_tot * nb) return;
    const long long inst = i / g.size_tot, n_t = i - inst * g.size_tot;
    int x[3];
    long long flat;
    const bool in = grid_coords(g, n_t, x, flat);
    wall_dist[i] = in ? dist[inst * g.n + flat] : (uint8_t)255;
}

// Selling's decomposition of n packed symmetric matrices in the planar layouts
// of the reference's VoronoiDecomposition kernel (Kernel_VoronoiDecomposition.h:45-69):
// m[c * n + p] (lower triangle, row major), weights[r * n + p],
// offsets[(i * SD + r) * n + p] for coordinate i of offset r.  Dimension 1: the
// weight is the matrix, the offset 1.  One thread per matrix, grid stride.
template <int D, class OffT>
__global__ void voronoi_kernel(const float *__restrict__ m, long long n, float *__restrict__ w,
                               OffT *__restrict__ e) {
    constexpr int SD = D * (D + 1) / 2;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        float mm[SD], ww[SD];
        int ee[SD][3];
#pragma unroll
        for (int c = 0; c < SD; ++c) mm[c] = __ldg(m + c * n + p);
        if constexpr (D == 1) {
            ww[0] = mm[0];
            ee[0][0] = 1;
        } else if constexpr (D == 2) {
            selling2(mm, ww, ee);
        } else {
            selling3(mm, ww, ee);
        }
#pragma unroll
        for (int r = 0; r < SD; ++r) {
            w[r * n + p] = ww[r];
#pragma unroll
            for (int i = 0; i < D; ++i) e[(i * SD + r) * n + p] = (OffT)ee[r][i];
        }
    }
}

template <int D>
static void launch_voronoi(const float *m, long long n, float *w, void *e, int offset_bytes, cudaStream_t st) {
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 32);
    switch (offset_bytes) {
        case 1: voronoi_kernel<D, int8_t><<<blocks, 256, 0, st>>>(m, n, w, static_cast<int8_t *>(e)); break;
        case 2: voronoi_kernel<D, int16_t><<<blocks, 256, 0, st>>>(m, n, w, static_cast<int16_t *>(e)); break;
        case 4: voronoi_kernel<D, int32_t><<<blocks, 256, 0, st>>>(m, n, w, static_cast<int32_t *>(e)); break;
        default: voronoi_kernel<D, int64_t><<<blocks, 256, 0, st>>>(m, n, w, static_cast<int64_t *>(e)); break;
    }
}

__global__ void selling_kernel(int nd, const float *m, int n, float *w, int *e) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float ww[6];
    int ee[6][3];
    if (nd == 2) {
        float mm[3] = {m[3 * p], m[3 * p + 1], m[3 * p + 2]};
        selling2(mm, ww, ee);
        for (int r = 0; r < 3; ++r) { w[3 * p + r] = ww[r]; e[(3 * p + r) * 2] = ee[r][0]; e[(3 * p + r) * 2 + 1] = ee[r][1]; }
    } else {
        float mm[6];
        for (int c = 0; c < 6; ++c) mm[c] = m[6 * p + c];
        selling3(mm, ww, ee);
        for (int r = 0; r < 6; ++r) { w[6 * p + r] = ww[r]; for (int c = 0; c < 3; ++c) e[(6 * p + r) * 3 + c] = ee[r][c]; }
    }
}

static inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace agd

using namespace agd;

extern "C" {

int agd_plan_create(const agd_instance *inst, int n, agd_plan **plan) {
    clear_error();
    return plan_create(inst, n, plan);
}

void agd_plan_destroy(agd_plan *plan) { delete plan; }

size_t agd_plan_workspace_bytes(const agd_plan *plan) { return plan ? plan->L.total : 0; }

int agd_plan_upload(const agd_plan *plan, void *workspace, size_t workspace_bytes, agd_stream_t stream) {
    clear_error();
    return plan_upload(plan, workspace, workspace_bytes, (cudaStream_t)stream);
}

int agd_plan_run(const agd_plan *plan, void *workspace, size_t workspace_bytes, agd_stats *stats,
                 const agd_launch *launch, agd_stream_t stream) {
    clear_error();
    return plan_run(plan, workspace, workspace_bytes, stats, launch, (cudaStream_t)stream);
}

size_t agd_eikonal_workspace_bytes(const agd_instance *inst, int n) {
    WsLayout L;
    if (!inst || n <= 0 || !layout(inst, n, L, static_cast<Inst *>(nullptr))) return 0;
    return L.total;
}

int agd_eikonal_solve(const agd_instance *inst, int n, void *workspace, size_t workspace_bytes, agd_stats *stats,
                      const agd_launch *launch, agd_stream_t stream) {
    clear_error();
    agd_plan *P = nullptr;
    int rc = plan_create(inst, n, &P);
    if (rc != AGD_STATUS_OK) return rc;
    rc = plan_upload(P, workspace, workspace_bytes, (cudaStream_t)stream);
    if (rc == AGD_STATUS_OK) rc = plan_run(P, workspace, workspace_bytes, stats, launch, (cudaStream_t)stream);
    delete P;
    return rc;
}

int agd_eikonal_solve_fixed_scratch(const agd_instance *inst, int n, agd_stats *stats, const agd_launch *launch,
                                    agd_stream_t stream) {
    clear_error();
    return fixed_scratch_solve(inst, n, stats, launch, (cudaStream_t)stream);
}

int agd_flow(const agd_instance *inst, float *flow_vector, float *flow_weightsum, float *flow_weights,
             int32_t *flow_indices, agd_stream_t stream) {
    clear_error();
    return flow_impl(inst, flow_vector, flow_weightsum, flow_weights, flow_indices, (cudaStream_t)stream);
}

int agd_prep_geom(int ndim, const int *shape, const int *shape_i, const float *metric, int broadcast, int is_dual,
                  const double *grid_scales, float *geom, agd_stream_t stream) {
    clear_error();
    Geo g;
    if (ndim < 2 || !geo_of(ndim, shape, shape_i, g) || !metric || !geom || !grid_scales)
        return set_error(AGD_STATUS_INVALID, "agd_prep_geom: bad arguments");
    prep_geom_kernel<<<blocks_for(g.size_tot, 256), 256, 0, (cudaStream_t)stream>>>(
        g, metric, broadcast, is_dual, grid_scales[0], grid_scales[1], ndim == 3 ? grid_scales[2] : 1.0, geom);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("prep_geom", err);
}

int agd_prep_geom_diagonal(int ndim, const int *shape, const int *shape_i, const float *costs, int broadcast,
                           int is_dual, const double *grid_scales, float *geom, agd_stream_t stream) {
    clear_error();
    Geo g;
    if (ndim < 1 || !geo_of(ndim, shape, shape_i, g) || !costs || !geom || !grid_scales)
        return set_error(AGD_STATUS_INVALID, "agd_prep_geom_diagonal: bad arguments");
    prep_diag_kernel<<<blocks_for(g.size_tot, 256), 256, 0, (cudaStream_t)stream>>>(
        g, costs, broadcast, is_dual, grid_scales[0], ndim > 1 ? grid_scales[1] : 1.0, ndim > 2 ? grid_scales[2] : 1.0,
        geom);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("prep_geom_diagonal", err);
}

int agd_prep_geom_rander(int ndim, const int *shape, const int *shape_i, const float *metric, int broadcast,
                         int is_dual, const double *grid_scales, float *geom, agd_stream_t stream) {
    clear_error();
    Geo g;
    if ((ndim != 2 && ndim != 3) || !geo_of(ndim, shape, shape_i, g) || !metric || !geom || !grid_scales)
        return set_error(AGD_STATUS_INVALID, "agd_prep_geom_rander: bad arguments");
    prep_rander_kernel<<<blocks_for(g.size_tot, 256), 256, 0, (cudaStream_t)stream>>>(
        g, metric, broadcast, is_dual, grid_scales[0], grid_scales[1], ndim == 3 ? grid_scales[2] : 1.0, geom);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("prep_geom_rander", err);
}

int agd_block_expand(int ndim, const int *shape, const int *shape_i, int nplanes, const float *src, int src_broadcast,
                     float pad, float *dst, agd_stream_t stream) {
    clear_error();
    Geo g;
    if (!geo_of(ndim, shape, shape_i, g) || nplanes < 1 || !src || !dst)
        return set_error(AGD_STATUS_INVALID, "agd_block_expand: bad arguments");
    block_expand_kernel<<<blocks_for(g.size_tot * nplanes, 256), 256, 0, (cudaStream_t)stream>>>(
        g, nplanes, src, src_broadcast, pad, dst);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("block_expand", err);
}

int agd_block_squeeze(int ndim, const int *shape, const int *shape_i, int nplanes, const float *src, float *dst,
                      agd_stream_t stream) {
    clear_error();
    Geo g;
    if (!geo_of(ndim, shape, shape_i, g) || nplanes < 1 || !src || !dst)
        return set_error(AGD_STATUS_INVALID, "agd_block_squeeze: bad arguments");
    block_squeeze_kernel<<<blocks_for(g.n * nplanes, 256), 256, 0, (cudaStream_t)stream>>>(g, nplanes, src, dst);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("block_squeeze", err);
}

int agd_prep_seeds(int ndim, const int *shape, const int *shape_i, const int32_t *seed_index, const float *seed_values,
                   int n, float *rhs, uint8_t *seedbits, uint8_t *trigger, agd_stream_t stream) {
    clear_error();
    Geo g;
    if (!geo_of(ndim, shape, shape_i, g) || n < 0 || (n > 0 && !seed_index) || (g.size_tot % 32) != 0)
        return set_error(AGD_STATUS_INVALID, "agd_prep_seeds: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    if (seedbits)
        seedbits_init_kernel<<<blocks_for(g.size_tot / 32, 256), 256, 0, st>>>(g, reinterpret_cast<unsigned *>(seedbits));
    if (trigger) cudaMemsetAsync(trigger, 0, (size_t)(g.size_tot / g.size_i), st);
    if (n > 0) {
        seeds_kernel<<<1, 32, 0, st>>>(g, seed_index, seed_values, n, rhs, reinterpret_cast<unsigned *>(seedbits),
                                       trigger, nullptr);
    }
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("prep_seeds", err);
}

int agd_prep_batch(const agd_batch_prep *p, agd_stream_t stream) {
    clear_error();
    Geo g;
    if (!p || (p->ndim != 2 && p->ndim != 3) || !geo_of(p->ndim, p->shape, p->shape_i, g) || p->n < 1 ||
        (g.size_tot % 32) != 0 || p->nseeds < 0 || (p->nseeds > 0 && !p->seed_index) || !p->rhs ||
        !p->values || !p->seedbits)
        return set_error(AGD_STATUS_INVALID, "agd_prep_batch: bad arguments");
    const int sd = p->ndim * (p->ndim + 1) / 2;
    int nmet = 0;
    switch (p->model) {
        case AGD_MODEL_ISOTROPIC: nmet = 0; break;
        case AGD_MODEL_RIEMANN: nmet = sd; break;
        case AGD_MODEL_DIAGONAL: nmet = p->ndim; break;
        case AGD_MODEL_RANDER: nmet = sd + p->ndim; break;
        default: return set_error(AGD_STATUS_INVALID, "agd_prep_batch: unknown model");
    }
    if (nmet && (!p->metric || !p->geom))
        return set_error(AGD_STATUS_INVALID,
                         "agd_prep_batch: Riemann, Diagonal and Rander instances need metric and geom");
    BatchPrep A;
    A.g = g;
    A.n = p->n;
    A.model = p->model;
    A.nmet = nmet;
    A.ngeom = nmet;  // the geometry planes of these models are as many as the metric's floats
    A.is_dual = p->is_dual;
    A.walls = p->walls;
    A.walls_stride = p->walls_shared ? 0 : g.n;
    A.trigger = p->trigger;
    A.size_o = g.size_tot / g.size_i;
    A.nseeds = p->nseeds;
    for (int k = 0; k < 3; ++k) A.h[k] = k < p->ndim ? (float)p->grid_scales[k] : 1.f;
    A.metric = p->metric;
    A.cost = p->cost;
    A.seed_values = p->seed_values;
    A.seed_index = p->seed_index;
    A.geom = p->geom;
    A.rhs = p->rhs;
    A.values = p->values;
    A.bits = reinterpret_cast<unsigned *>(p->seedbits);
    A.bad = p->bad_seed;
    if (g.size_tot >= (1ll << 31) || p->n > 65535)
        return set_error(AGD_STATUS_INVALID, "agd_prep_batch: at most 65535 instances of fewer than 2^31 points");
    bool pow2 = true;
    for (int k = 0; k < 3; ++k) {
        int l = 0;
        while ((1 << l) < g.si[k]) ++l;
        A.si_log2[k] = l;
        pow2 = pow2 && (1 << l) == g.si[k];
    }
    if (!pow2) A.si_log2[0] = A.si_log2[1] = A.si_log2[2] = -1;
    cudaStream_t st = (cudaStream_t)stream;
    // about 16 resident 256-thread blocks per SM over all the instances
    const long long per_inst = std::max<long long>(1, 148LL * 16 / p->n);
    const dim3 grid((unsigned)std::min<long long>((g.size_tot + 255) / 256, per_inst), (unsigned)p->n);
    prep_batch_kernel<<<grid, 256, 0, st>>>(A);
    if (p->nseeds > 0) seeds_batch_kernel<<<blocks_for(p->n, 128), 128, 0, st>>>(A);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("prep_batch", err);
}

int agd_prep_walls(int ndim, const int *shape, const int *shape_i, const uint8_t *walls, int bound, uint8_t *wall_dist,
                   uint8_t *tmp, float *rhs, uint8_t *seedbits, agd_stream_t stream) {
    clear_error();
    Geo g;
    if ((ndim != 2 && ndim != 3) || !shape || !shape_i || !geo_of(ndim, shape, shape_i, g) || (g.size_tot % 32) != 0 ||
        !walls || !wall_dist || !tmp || bound < 0 || bound > 254)
        return set_error(AGD_STATUS_INVALID, "agd_prep_walls: bad arguments (bound in [0, 254])");
    cudaStream_t st = (cudaStream_t)stream;
    // _SetGeometry.py:271-277: 0 at walls, `bound` passes of the L1 kernel, cut beyond `bound`
    const int rc = distance_map(ndim, shape, walls, bound, bound, true, tmp, tmp + g.n, st);
    if (rc != AGD_STATUS_OK) return rc;
    walls_kernel<<<(unsigned)((g.size_tot + 255) / 256), 256, 0, st>>>(g, walls, tmp, wall_dist, rhs,
                                                                       reinterpret_cast<unsigned *>(seedbits));
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("prep_walls", err);
}

int agd_prep_walls_batch(int ndim, const int *shape, const int *shape_i, int n, const uint8_t *walls, int bound,
                         uint8_t *wall_dist, uint8_t *tmp, agd_stream_t stream) {
    clear_error();
    Geo g;
    if ((ndim != 2 && ndim != 3) || !shape || !shape_i || !geo_of(ndim, shape, shape_i, g) || n < 1 || !walls ||
        !wall_dist || !tmp || bound < 0 || bound > 254)
        return set_error(AGD_STATUS_INVALID, "agd_prep_walls_batch: bad arguments (bound in [0, 254])");
    cudaStream_t st = (cudaStream_t)stream;
    const long long np = g.n * n;  // grid points of all the instances
    const int rc = distance_map(ndim, shape, walls, bound, bound, true, tmp, tmp + np, st, n);
    if (rc != AGD_STATUS_OK) return rc;
    wall_dist_batch_kernel<<<blocks_for(g.size_tot * n, 256), 256, 0, st>>>(g, n, tmp, wall_dist);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("prep_walls_batch", err);
}

int agd_voronoi_decomposition(int ndim, const float *m, long long n, float *weights, void *offsets, int offset_bytes,
                              agd_stream_t stream) {
    clear_error();
    if (ndim < 1 || ndim > 3 || n < 0 || (n > 0 && (!m || !weights || !offsets)) ||
        (offset_bytes != 1 && offset_bytes != 2 && offset_bytes != 4 && offset_bytes != 8))
        return set_error(AGD_STATUS_INVALID, "agd_voronoi_decomposition: bad arguments (ndim 1 to 3, "
                                             "offset_bytes 1, 2, 4 or 8)");
    if (n == 0) return AGD_STATUS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (ndim == 1) launch_voronoi<1>(m, n, weights, offsets, offset_bytes, st);
    else if (ndim == 2) launch_voronoi<2>(m, n, weights, offsets, offset_bytes, st);
    else launch_voronoi<3>(m, n, weights, offsets, offset_bytes, st);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("voronoi_decomposition", err);
}

int agd_selling(int ndim, const float *m, int n, float *weights, int32_t *offsets, agd_stream_t stream) {
    clear_error();
    if ((ndim != 2 && ndim != 3) || n < 0 || (n > 0 && (!m || !weights || !offsets)))
        return set_error(AGD_STATUS_INVALID, "agd_selling: bad arguments");
    if (n == 0) return AGD_STATUS_OK;
    selling_kernel<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(ndim, m, n, weights, offsets);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("selling", err);
}

}  // extern "C"
