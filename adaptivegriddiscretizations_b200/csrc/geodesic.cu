// Geodesic backtracking on B200: the distance-to-seed map used by the stopping
// criteria, and the midpoint ODE on the upwind flow, one warp per tip.
//
// The reference runs its GeodesicODE kernel in chunks of `typical_len` steps
// and restarts each unfinished geodesic from its last point on the host
// (agd/Eikonal/HFM_CUDA/_GetGeodesics.py:111-134).  Here a warp runs all of
// its chunks in one launch; a chunk boundary resets the same state the
// reference's restart resets (stopping-criteria history, cell cache), so the
// paths are the reference's.  The stepping follows
// cuda/Kernel_GeodesicODE.h:164-412 with the precomputed flow of
// GeodesicODE_Opt.h:236-245, in float.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "agd_common.cuh"
#include "agd_internal.h"

namespace agd {

// ------------------------------------------------------ distance to seeds ---
struct EGeo {
    int nd, shape[3];
    long long n;  // points of one instance
    int nb;       // instances, one after the other
};

// One min-plus pass: out(x) = min over the 3^d neighbours y of min(255, in(y) + k(y - x)),
// k = round(5 |y - x|) (inf_convolution with distance_kernel(1, ndim, uint8, mult=5)),
// or with l1, k = |y - x|_1 (distance_kernel(1, ndim, uint8, ord=1)).
// FROM_MASK: `in` is the mask, read as 0 at its points and 255 elsewhere (the
// first pass); CUT: values above `cut` become 255 (the last pass).
// Threads run along the last axis, blocks stride over the rows of the others.
template <int D, bool FROM_MASK, bool CUT>
__global__ void __launch_bounds__(256) infconv_kernel(EGeo g, const uint8_t *__restrict__ in, int l1, int cut,
                                                      uint8_t *__restrict__ out) {
    constexpr int NK = D == 2 ? 9 : 27;
    const int nlast = g.shape[D - 1];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nlast) return;
    const long long nrows = g.n / nlast;
    long long stride[D];
    stride[D - 1] = 1;
    for (int k = D - 2; k >= 0; --k) stride[k] = stride[k + 1] * g.shape[k + 1];
    // rows of all the instances; a neighbour is one of the same instance
    for (long long r = blockIdx.y * (long long)blockDim.y + threadIdx.y; r < nrows * g.nb;
         r += (long long)gridDim.y * blockDim.y) {
        const long long rr = r % nrows;  // row within the instance
        int x[D];
        x[D - 1] = c;
        if (D == 3) {
            x[0] = (int)(rr / g.shape[1]);
            x[1] = (int)(rr - (long long)x[0] * g.shape[1]);
        } else {
            x[0] = (int)rr;
        }
        const long long p = r * nlast + c;
        int best = 255;
#pragma unroll
        for (int ic = 0; ic < NK; ++ic) {
            int n2 = 0;
            bool ok = true;
            long long m = p;
#pragma unroll
            for (int k = 0, q = ic; k < D; ++k, q /= 3) {
                const int o = q % 3 - 1;
                n2 += o * o;
                const int y = x[k] + o;
                ok = ok && y >= 0 && y < g.shape[k];
                m += o * stride[k];
            }
            if (!ok) continue;
            // offsets in {-1, 0, 1}^d: |o|_1 = |o|^2; round(5 |o|) = 0, 5, 7, 9
            const int kv = l1 ? n2 : (n2 == 0 ? 0 : (n2 == 1 ? 5 : (n2 == 2 ? 7 : 9)));
            const int a = FROM_MASK ? (in[m] ? 0 : 255) : in[m];
            best = min(best, (a >= 255 - kv) ? 255 : a + kv);
        }
        if (CUT && best > cut) best = 255;
        out[p] = (uint8_t)best;
    }
}

template <int D>
static void infconv_pass(const EGeo &g, const uint8_t *in, bool from_mask, bool cut_it, int l1, int cut,
                         uint8_t *out, cudaStream_t st) {
    const dim3 block(32, 8);
    const long long nrows = g.n / g.shape[D - 1] * g.nb;
    const dim3 grid((unsigned)((g.shape[D - 1] + 31) / 32), (unsigned)std::min<long long>((nrows + 7) / 8, 16384));
    if (from_mask && cut_it) infconv_kernel<D, true, true><<<grid, block, 0, st>>>(g, in, l1, cut, out);
    else if (from_mask) infconv_kernel<D, true, false><<<grid, block, 0, st>>>(g, in, l1, cut, out);
    else if (cut_it) infconv_kernel<D, false, true><<<grid, block, 0, st>>>(g, in, l1, cut, out);
    else infconv_kernel<D, false, false><<<grid, block, 0, st>>>(g, in, l1, cut, out);
}

__global__ void eucl_init_kernel(EGeo g, const uint8_t *mask, uint8_t *out) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p < g.n * g.nb) out[p] = mask[p] ? 0 : 255;
}

__global__ void eucl_cut_kernel(EGeo g, const uint8_t *in, int cut, uint8_t *out) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p < g.n * g.nb) out[p] = in[p] > cut ? 255 : in[p];
}

// ------------------------------------------------------------ geodesics ---
enum { kContinue = 0, kAtSeed, kInWall, kStationnary, kPastSeed, kVanishingFlow };

struct GeoArgs {
    int nd;
    int shape[3], shape_i[3], shape_o[3];
    int size_i;
    long long size_tot;
    const float *u, *fvec, *fwsum;
    const uint8_t *eucl;
    const float *tips;
    int ntips;
    float step, causality;
    int typical_len, max_chunks, eucl_delay, nymin_delay, pastseed_delay;
    float *paths;
    int cap;
    int *lengths;
    int8_t *stops;
};

constexpr int kMaxHist = 256;  // bound on 1 + max(eucl_delay, nymin_delay)

// The point data around the current cell, in shared memory, one per warp: the
// values, flow weight sums, flow planes and distance-to-seed bytes of a W^D
// box of grid points, with the stopping criteria's history.  A warp traces one
// geodesic; its 32 lanes fill the box together (asynchronous 4-byte copies for
// the floats, batched loads for the bytes), and then all of them step the same
// ODE on the same data, so that the control flow stays warp-uniform and the
// steps read shared memory instead of waiting on global loads.  The box is
// refilled, centred on the current cell, when a cell leaves it: after at least
// W/2 - 1 points of travel.
template <int D>
struct GeoWindow {
    static constexpr int W = D == 2 ? 32 : 12;
    static constexpr int WT = D == 2 ? W * W : W * W * W;
    static constexpr int NJ = WT / 32;  // points per lane
    static_assert(WT % 32 == 0, "whole warps of points");
    float u[WT], wsum[WT], flow[D][WT];
    uint8_t eucl[WT];
    int org[D];
    int tq[D][W], tr[D][W];  // per axis: tile and in-tile coordinate of org + t, tq -1 outside the grid
    long long nymin_p[kMaxHist];
    uint8_t eucl_p[kMaxHist];
};

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int D>
struct Walker {
    using Win = GeoWindow<D>;
    static constexpr int NC = 1 << D;
    static constexpr int W = Win::W;
    const GeoArgs A;  // a copy: the fields stay in registers
    Win &S;
    const int lane;
    int xq[D];
    long long nymin;  // grid index of the retained corner (the reference keeps its
                      // bilevel index: the same point, so the same equality tests)
    int eucl_min;     // distance-to-seed byte at that corner
    float thr;
    float flow_c[NC][D], dist_c[NC], wsum_c[NC];

    __device__ __forceinline__ Walker(const GeoArgs &a, Win &s, int ln) : A(a), S(s), lane(ln) { reset(); }
    __device__ __forceinline__ void reset() {
        for (int k = 0; k < D; ++k) xq[k] = kIntMax;
        nymin = -1;
        eucl_min = 255;
        thr = 0.f;
    }
    __device__ __forceinline__ bool inside(const int *y) const {
        for (int k = 0; k < D; ++k)
            if (y[k] < 0 || y[k] >= A.shape[k]) return false;
        return true;
    }
    __device__ __forceinline__ long long gridindex(const int *y) const {
        long long n = 0;
        for (int k = 0; k < D; ++k) n = n * A.shape[k] + y[k];
        return n;
    }
    // Position in the box of a grid point that it holds.  When the cell
    // xq..xq+1 passes covers(), a corner that is inside the grid has box
    // coordinates in [0, W) on every axis.
    __device__ __forceinline__ int local(const int *y) const {
        int li = 0;
        for (int k = 0; k < D; ++k) li = li * W + (y[k] - S.org[k]);
        return li;
    }
    __device__ __forceinline__ bool covers() const {
        bool ok = true;
        for (int k = 0; k < D; ++k) ok = ok && xq[k] >= S.org[k] && xq[k] < S.org[k] + (W - 1);
        return ok;
    }
    // Refill the box around the cell at xq (all lanes, warp-uniform).
    __device__ __forceinline__ void fill() {
        __syncwarp();  // every lane has finished reading the previous box
        int org[D];
        for (int k = 0; k < D; ++k) org[k] = xq[k] - (W / 2 - 1);
        if (lane < W) {
            for (int k = 0; k < D; ++k) {
                const int y = org[k] + lane;
                const bool in = y >= 0 && y < A.shape[k];
                S.tq[k][lane] = in ? y / A.shape_i[k] : -1;
                S.tr[k][lane] = in ? y % A.shape_i[k] : 0;
            }
        }
        if (lane == 0)
            for (int k = 0; k < D; ++k) S.org[k] = org[k];
        __syncwarp();
        constexpr int G = 16;  // byte loads in flight per lane
#pragma unroll 1
        for (int j0 = 0; j0 < Win::NJ; j0 += G) {
            int e[G];
#pragma unroll
            for (int jj = 0; jj < G; ++jj) {
                e[jj] = 255;
                const int j = j0 + jj;
                if (j >= Win::NJ) continue;
                const int p = j * 32 + lane;
                int t[D], r = p;
                for (int k = D - 1; k >= 0; --k) { t[k] = r % W; r /= W; }
                bool in = true;
                long long n_o = 0, g = 0;
                int n_i = 0;
                for (int k = 0; k < D; ++k) {
                    const int q = S.tq[k][t[k]];
                    in = in && q >= 0;
                    n_o = n_o * A.shape_o[k] + q;
                    n_i = n_i * A.shape_i[k] + S.tr[k][t[k]];
                    g = g * A.shape[k] + (org[k] + t[k]);
                }
                if (!in) continue;
                const long long n = n_o * A.size_i + n_i;
                cp_async4(&S.u[p], A.u + n);
                cp_async4(&S.wsum[p], A.fwsum + n);
                for (int k = 0; k < D; ++k) cp_async4(&S.flow[k][p], A.fvec + k * A.size_tot + n);
                e[jj] = __ldg(A.eucl + g);
            }
#pragma unroll
            for (int jj = 0; jj < G; ++jj)
                if (j0 + jj < Win::NJ) S.eucl[(j0 + jj) * 32 + lane] = (uint8_t)e[jj];
        }
        cp_async_wait_all();
        __syncwarp();
    }
    // Kernel_GeodesicODE.h:164-260 (NormalizedFlow)
    __device__ __forceinline__ int normalized_flow(const float *x, float *flow) {
        bool newcell = false;
        for (int k = 0; k < D; ++k) {
            const int q = (int)floorf(x[k]);
            if (q != xq[k]) newcell = true;
            xq[k] = q;
        }
        float dx[D], wts[NC];
        for (int k = 0; k < D; ++k) dx[k] = x[k] - (float)xq[k];
        for (int i = 0; i < NC; ++i) {
            float w = 1.f;
            for (int k = 0; k < D; ++k) w *= ((i >> k) & 1) ? dx[k] : 1.f - dx[k];
            wts[i] = w;
        }
        if (newcell) {
            if (!covers()) fill();
            for (int i = 0; i < NC; ++i) {
                int y[D];
                for (int k = 0; k < D; ++k) y[k] = xq[k] + ((i >> k) & 1);
                if (!inside(y)) {
                    dist_c[i] = finf();
                    continue;
                }
                const int li = local(y);
                dist_c[i] = S.u[li];
                wsum_c[i] = S.wsum[li];
                for (int k = 0; k < D; ++k) flow_c[i][k] = S.flow[k][li];
            }
            float dmin = finf(), ws = 0.f;
            int imin = 0;
            const float wthr = 0.5f / NC;
            for (int i = 0; i < NC; ++i) {
                if (wts[i] < wthr) continue;
                if (dist_c[i] < dmin) { imin = i; dmin = dist_c[i]; ws = wsum_c[i]; }
            }
            if (dmin == finf()) return kInWall;
            int y[D];
            for (int k = 0; k < D; ++k) y[k] = xq[k] + ((imin >> k) & 1);
            nymin = gridindex(y);
            eucl_min = S.eucl[local(y)];
            if (ws == 0.f) return kAtSeed;
            thr = dmin + A.causality / ws;
        }
        for (int k = 0; k < D; ++k) flow[k] = 0.f;
        for (int i = 0; i < NC; ++i) {
            if (dist_c[i] >= thr) continue;
            for (int k = 0; k < D; ++k) flow[k] += wts[i] * flow_c[i][k];
        }
        float n2 = 0.f;
        for (int k = 0; k < D; ++k) n2 += flow[k] * flow[k];
        const float nrm = sqrtf(n2);
        if (!(nrm > 0.f)) return kVanishingFlow;
        // The correctly rounded float reciprocal: the reference divides in
        // double and rounds to float, which gives the same value (a double
        // quotient has more than 2 x 24 + 2 bits, so the second rounding is
        // innocuous).
        const float l = __frcp_rn(nrm);
        for (int k = 0; k < D; ++k) flow[k] *= l;
        return kContinue;
    }
};

// One warp per tip.
template <int D>
__global__ void __launch_bounds__(32) geodesic_kernel(GeoArgs A) {
    __shared__ GeoWindow<D> S;
    const int tip = blockIdx.x;
    const int lane = threadIdx.x;
    if (tip >= A.ntips) return;
    float *out = A.paths + (long long)tip * A.cap * D;
    float x[D];
    for (int k = 0; k < D; ++k) x[k] = A.tips[tip * D + k];
    if (lane == 0)
        for (int k = 0; k < D; ++k) out[k] = x[k];
    if (lane < D) S.org[lane] = kIntMax / 2;  // an empty box: the first cell fills it
    __syncwarp();
    int pos = 1, stop = kContinue;
    const int hlen = 1 + max(A.eucl_delay, A.nymin_delay);
    Walker<D> Wk(A, S, lane);
    for (int chunk = 0; chunk < A.max_chunks; ++chunk) {
        // a chunk starts afresh from the last point, as the reference's restart does
        for (int l = lane; l < hlen; l += 32) {
            S.eucl_p[l] = 255;
            S.nymin_p[l] = -1;
        }
        __syncwarp();
        Wk.reset();
        // the PastSeed test waits pastseed_delay steps in the first chunk only
        // (_GetGeodesics.py:107-109,133)
        const int ps_delay = chunk == 0 ? A.pastseed_delay : 0;
        int l = 1 % hlen;  // len % hlen
        int len;
        for (len = 1; len < A.typical_len; ++len) {
            float xp[D], xm[D], flow[D];
            for (int k = 0; k < D; ++k) xp[k] = x[k];
            stop = Wk.normalized_flow(x, flow);
            if (stop != kContinue) break;
            // every lane holds the same values: the history is written alike by
            // all, once every lane has read the previous step's entries
            __syncwarp();
            S.nymin_p[l] = Wk.nymin;
            S.eucl_p[l] = (uint8_t)Wk.eucl_min;
            __syncwarp();
            int ln = l - A.nymin_delay, le = l - A.eucl_delay;
            if (ln < 0) ln += hlen;
            if (le < 0) le += hlen;
            if (Wk.nymin == S.nymin_p[ln]) { stop = kStationnary; break; }
            // The reference's subscript is a boolean expression (cuda/Kernel_GeodesicODE.h:331).
            const int cmp = (le != 0) && (len >= ps_delay);
            if (S.eucl_p[l] > S.eucl_p[cmp]) { stop = kPastSeed; break; }
            for (int k = 0; k < D; ++k) xm[k] = (0.5f * A.step) * flow[k] + xp[k];
            stop = Wk.normalized_flow(xm, flow);
            if (stop != kContinue) break;
            for (int k = 0; k < D; ++k) x[k] = A.step * flow[k] + xp[k];
            if (pos < A.cap) {
                if (lane == 0)
                    for (int k = 0; k < D; ++k) out[pos * D + k] = x[k];
                ++pos;
            }
            l = l + 1 == hlen ? 0 : l + 1;
        }
        if (stop != kContinue) break;
        __syncwarp();  // the history is reset only once every lane has read it
    }
    if (lane == 0) {
        A.lengths[tip] = pos;
        A.stops[tip] = (int8_t)stop;
    }
}

static inline unsigned nblocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// Min-plus distance map in grid layout: 0 at the mask points, 255 elsewhere,
// then `npasses` passes of infconv_kernel and values above `cut` set to 255.
// The first pass reads the mask and the last one applies the cut; the passes
// alternate between `out` and `tmp` so that the last one writes `out`.
// nb instances one after the other, each its own map.  tmp: scratch of nb
// prod(shape) bytes.
int distance_map(int ndim, const int *shape, const uint8_t *mask, int npasses, int cut, bool l1, uint8_t *out,
                 uint8_t *tmp, cudaStream_t st, int nb) {
    if ((ndim != 2 && ndim != 3) || !shape || !mask || !out || !tmp || npasses < 0 || nb < 1)
        return set_error(AGD_STATUS_INVALID, "distance map: bad arguments");
    EGeo g;
    g.nd = ndim;
    g.nb = nb;
    g.n = 1;
    for (int k = 0; k < 3; ++k) g.shape[k] = 1;
    for (int k = 0; k < ndim; ++k) {
        if (shape[k] <= 0) return set_error(AGD_STATUS_INVALID, "distance map: bad shape");
        g.shape[k] = shape[k];
        g.n *= shape[k];
    }
    const int bs = 256;
    if (npasses == 0) {
        eucl_init_kernel<<<nblocks(g.n * nb, bs), bs, 0, st>>>(g, mask, tmp);
        eucl_cut_kernel<<<nblocks(g.n * nb, bs), bs, 0, st>>>(g, tmp, cut, out);
    } else {
        const uint8_t *src = mask;
        for (int it = 0; it < npasses; ++it) {
            uint8_t *dst = ((npasses - 1 - it) % 2 == 0) ? out : tmp;
            if (ndim == 2) infconv_pass<2>(g, src, it == 0, it == npasses - 1, l1 ? 1 : 0, cut, dst, st);
            else infconv_pass<3>(g, src, it == 0, it == npasses - 1, l1 ? 1 : 0, cut, dst, st);
            src = dst;
        }
    }
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("distance map", err);
}

}  // namespace agd

using namespace agd;

extern "C" {

int agd_eucl_map(int ndim, const int *shape, const uint8_t *seed_mask, int npasses, int cut, uint8_t *eucl,
                 uint8_t *tmp, agd_stream_t stream) {
    clear_error();
    return distance_map(ndim, shape, seed_mask, npasses, cut, false, eucl, tmp, (cudaStream_t)stream);
}

int agd_geodesics(const agd_instance *inst, const float *flow_vector, const float *flow_weightsum, const uint8_t *eucl,
                  const float *tips, int ntips, float step, float causality, int typical_len, int max_chunks,
                  int eucl_delay, int nymin_delay, int pastseed_delay, float *paths, int cap, int32_t *lengths,
                  int8_t *stops, agd_stream_t stream) {
    clear_error();
    if (!inst || (inst->ndim != 2 && inst->ndim != 3) || ntips < 0 || !flow_vector || !flow_weightsum || !eucl ||
        !inst->values || typical_len < 2 || max_chunks < 1 || eucl_delay < 0 || nymin_delay < 0 || pastseed_delay < 0 ||
        1 + (eucl_delay > nymin_delay ? eucl_delay : nymin_delay) > kMaxHist || cap < 1 ||
        (ntips > 0 && (!tips || !paths || !lengths || !stops)))
        return set_error(AGD_STATUS_INVALID, "agd_geodesics: bad arguments");
    if (ntips == 0) return AGD_STATUS_OK;
    GeoArgs A;
    A.nd = inst->ndim;
    A.size_i = 1;
    long long so = 1;
    for (int k = 0; k < 3; ++k) { A.shape[k] = A.shape_i[k] = A.shape_o[k] = 1; }
    for (int k = 0; k < A.nd; ++k) {
        if (inst->shape[k] <= 0 || inst->shape_i[k] <= 0) return set_error(AGD_STATUS_INVALID, "bad shape");
        A.shape[k] = inst->shape[k];
        A.shape_i[k] = inst->shape_i[k];
        A.shape_o[k] = (inst->shape[k] + inst->shape_i[k] - 1) / inst->shape_i[k];
        A.size_i *= inst->shape_i[k];
        so *= A.shape_o[k];
    }
    A.size_tot = so * A.size_i;
    A.u = inst->values;
    A.fvec = flow_vector;
    A.fwsum = flow_weightsum;
    A.eucl = eucl;
    A.tips = tips;
    A.ntips = ntips;
    A.step = step;
    A.causality = causality;
    A.typical_len = typical_len;
    A.max_chunks = max_chunks;
    A.eucl_delay = eucl_delay;
    A.nymin_delay = nymin_delay;
    A.pastseed_delay = pastseed_delay;
    A.paths = paths;
    A.cap = cap;
    A.lengths = lengths;
    A.stops = stops;
    // one warp per geodesic, one geodesic per block: the tips spread over the SMs
    if (A.nd == 2) geodesic_kernel<2><<<(unsigned)ntips, 32, 0, (cudaStream_t)stream>>>(A);
    else geodesic_kernel<3><<<(unsigned)ntips, 32, 0, (cudaStream_t)stream>>>(A);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? AGD_STATUS_OK : set_cuda_error("geodesics", err);
}

}  // extern "C"
