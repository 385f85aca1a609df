// Forward and reverse-mode differentiation of the eikonal solution on B200.
//
// Linearising sum_k w_k (u - v_k)_+^2 = c^2 at the solution gives, at every
// non-seed point x, diag(x) du(x) - sum_k fw_k(x) du(y_k(x)) = r(x), where
// fw_k are the upwind flow weights, y_k(x) the upwind neighbours and diag the
// weight sum (1 at seeds and outside the domain).  The forward mode solves it
// for r = c dc (dc a variation of the cost; r is the seed value's variation at
// a seed); the reverse mode solves the transposed system
// diag(x) lam(x) - sum_{z: y_k(z) = x} fw_k(z) lam(z) = s(x)
// (agd/Eikonal/HFM_CUDA/_PostProcess.py:155-219).
//
// The reference transposes the graph with an iterative claim loop relaunched
// from the host (graph_reverse.py:10-77, cuda/GraphReverse.h:35-82) and solves
// with the block Gauss-Seidel kernel of cuda/Kernel_LinearUpdate.h under the
// adaptive Gauss-Seidel tile schedule.  Here: a counting-sort CSR transpose
// (rows sorted, so sums are deterministic), then the tile scheduler of the
// eikonal solver with a linear tile visit.  Every tile is visited at the first
// epoch; afterwards a point whose value moved activates exactly the tiles of
// the points that depend on it (reverse: its upwind neighbours; forward: the
// points it is an upwind neighbour of, from the transpose), so dependencies
// that skip over tiles are never missed.
#include <cuda_runtime.h>

#include <cstdio>

#include "sched.cuh"

namespace agd {

// ------------------------------------------------------------ transpose ---
struct RevGeom {
    long long size_tot;
    int nact;
};

__global__ void rev_count_kernel(RevGeom g, const float *fw, const int *fidx, int *count) {
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.size_tot) return;
    for (int k = 0; k < g.nact; ++k) {
        const float w = fw[k * g.size_tot + n];
        const int y = fidx[k * g.size_tot + n];
        if (w != 0.f && y >= 0 && y < g.size_tot) atomicAdd(count + y, 1);
    }
}

__global__ void rev_fill_kernel(RevGeom g, const float *fw, const int *fidx, const int *rowptr, int *cursor, int *src,
                                float *wt) {
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.size_tot) return;
    for (int k = 0; k < g.nact; ++k) {
        const float w = fw[k * g.size_tot + n];
        const int y = fidx[k * g.size_tot + n];
        if (w != 0.f && y >= 0 && y < g.size_tot) {
            const int pos = rowptr[y] + atomicAdd(cursor + y, 1);
            src[pos] = (int)n;
            wt[pos] = w;
        }
    }
}

// Rows in increasing source order: the fill order depends on the schedule.
// A row of up to kSortRegs entries is sorted in registers (an insertion
// network with fixed indices, strict comparisons as below); longer rows in
// place in global memory.
constexpr int kSortRegs = 12;
__global__ void rev_sort_kernel(RevGeom g, const int *rowptr, int *src, float *wt) {
    const long long y = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (y >= g.size_tot) return;
    const int a = rowptr[y], b = rowptr[y + 1];
    const int len = b - a;
    if (len <= 1) return;
    if (len <= kSortRegs) {
        int sr[kSortRegs];
        float wr[kSortRegs];
#pragma unroll
        for (int i = 0; i < kSortRegs; ++i)
            if (i < len) {
                sr[i] = src[a + i];
                wr[i] = wt[a + i];
            }
#pragma unroll
        for (int i = 1; i < kSortRegs; ++i) {
#pragma unroll
            for (int j = i; j > 0; --j) {
                if (i < len && sr[j - 1] > sr[j]) {
                    const int ts = sr[j - 1];
                    sr[j - 1] = sr[j];
                    sr[j] = ts;
                    const float tw = wr[j - 1];
                    wr[j - 1] = wr[j];
                    wr[j] = tw;
                }
            }
        }
#pragma unroll
        for (int i = 0; i < kSortRegs; ++i)
            if (i < len) {
                src[a + i] = sr[i];
                wt[a + i] = wr[i];
            }
        return;
    }
    for (int i = a + 1; i < b; ++i) {
        const int s = src[i];
        const float w = wt[i];
        int j = i - 1;
        while (j >= a && src[j] > s) {
            src[j + 1] = src[j];
            wt[j + 1] = wt[j];
            --j;
        }
        src[j + 1] = s;
        wt[j + 1] = w;
    }
}

// Exclusive scan of n ints in three passes (blocks of 1024, block totals, offsets).
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ int block_excl_scan(int v, int *tot) {
    __shared__ int ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int inc = warp_incl_scan(v, lane);
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        int x = lane < nw ? ws[lane] : 0;
        x = warp_incl_scan(x, lane);
        if (lane < nw) ws[lane] = x;
    }
    __syncthreads();
    const int off = warp > 0 ? ws[warp - 1] : 0;
    if (tot) *tot = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return off + inc - v;
}

__global__ void scan_blocks_kernel(const int *in, int *out, long long n, int *block_tot) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    int tot;
    const int ex = block_excl_scan(v, &tot);
    if (i < n) out[i] = ex;
    if (threadIdx.x == 0) block_tot[blockIdx.x] = tot;
}

__global__ void scan_totals_kernel(int *block_tot, int nb, int *grand) {
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? block_tot[i] : 0;
        int tot;
        const int ex = block_excl_scan(v, &tot);
        if (i < nb) block_tot[i] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *grand = carry;
}

__global__ void scan_add_kernel(int *out, long long n, const int *block_off) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] += block_off[blockIdx.x];
}

// ----------------------------------------------------------- linear visit ---
struct LinArgs {
    const int *rowptr, *src;
    const float *wt;
    const float *wsum, *sens;
    float *lam;
    const float *fw;
    const int *fidx;
    int nact;
    float atol, rtol;
};

// FWD: rows from the forward flow planes (fw, fidx), activation through the
// transpose (rowptr, src); reverse: rows from the transpose, activation
// through the forward planes.
template <int SIZE, bool FWD>
struct LinearVisitor {
    static constexpr int P = SIZE / 32;
    static constexpr int kMaxSweeps = 4 * SIZE;  // in-tile chains are shorter than the tile
    using Args = LinArgs;
    // In-tile entries of each point's row, kept for the sweeps: weight and
    // in-tile index of up to K of them, in row order (a row with more goes on
    // reading the rest from global memory).  Without this cache every sweep
    // re-read the rows through L2: 4.3 us a sweep, 70 % of a visit at 200^3.
    static constexpr int K = SIZE == 256 ? 4 : 8;
    static constexpr int kRowUnroll = K < 6 ? K : 6;  // row entries unrolled in the init (nact <= 6)
    struct Smem {
        float l[SIZE];
        float cw[K][SIZE];
        unsigned char cz[K][SIZE];
    };
    static cudaError_t prepare(const Sched &, const WsLayout &, cudaStream_t) { return cudaSuccess; }
    static cudaError_t finalize(const Sched &, const WsLayout &, cudaStream_t) { return cudaSuccess; }
    // Resident CTAs per SM: the reverse worker fits 64 registers with 20 bytes of
    // spills (8 CTAs: -3 % time per Riemann3 200^3 call against 6 at 80
    // registers), the forward one 72 registers (7 CTAs).
    static constexpr int kMinCtas = SIZE == 256 ? 4 : (FWD ? 7 : 8);
    // A linear solve is usually one large instance: its epochs (~15 k tiles at
    // 200^3) are published in batches; the worker's registers stay within the
    // kMinCtas budget.
    static constexpr bool kBulkPublish = true;
    static constexpr bool kBatchScheduling = false;

    __device__ static void visit(const Sched &S, const Args &A, int t, int ii, int e, int lane, Smem &sm) {
        const Inst &I = S.inst[ii];
        const int n_o = t - I.tile_base;
        const long long base = (long long)n_o * SIZE;
        float old[P], diag[P], acc[P];
        int r0[P], r1[P];
        unsigned cnt = 0, ovf = 0;  // per point p: cached entries (4 bits at 4p), more than K (bit p)
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int n_i = lane + 32 * p;
            const long long n_t = base + n_i;
            old[p] = __ldcg(A.lam + n_t);
            sm.l[n_i] = old[p];
            const float d = __ldg(A.wsum + n_t);
            diag[p] = d == 0.f ? 1.f : d;
            float a = __ldg(A.sens + n_t);
            r0[p] = __ldg(A.rowptr + n_t);
            r1[p] = __ldg(A.rowptr + n_t + 1);
            int c = 0;
            // Out-of-tile entries are summed once per visit, in row order; the
            // in-tile ones are cached.  The first kRowUnroll entries of a row are
            // unrolled so that their loads are issued together: a row walked
            // one entry at a time costs two dependent L2 round trips per entry.
            if constexpr (FWD) {
#pragma unroll
                for (int k = 0; k < kRowUnroll; ++k) {  // upwind neighbours: nact <= kRowUnroll
                    if (k >= A.nact) continue;
                    const float w = __ldg(A.fw + k * I.size_tot + n_t);
                    const int y = __ldg(A.fidx + k * I.size_tot + n_t);
                    if (w == 0.f || y < 0 || (long long)y >= I.size_tot) continue;
                    if ((long long)y / SIZE != n_o) {
                        a += w * __ldcg(A.lam + y);
                    } else {  // c <= k < K
                        sm.cw[c][n_i] = w;
                        sm.cz[c][n_i] = (unsigned char)(y - (int)base);
                        ++c;
                    }
                }
                for (int k = kRowUnroll; k < A.nact; ++k) {  // more neighbours than the unrolled part
                    const float w = __ldg(A.fw + k * I.size_tot + n_t);
                    const int y = __ldg(A.fidx + k * I.size_tot + n_t);
                    if (w == 0.f || y < 0 || (long long)y >= I.size_tot) continue;
                    if ((long long)y / SIZE != n_o) {
                        a += w * __ldcg(A.lam + y);
                    } else if (c < K) {
                        sm.cw[c][n_i] = w;
                        sm.cz[c][n_i] = (unsigned char)(y - (int)base);
                        ++c;
                    } else {
                        ovf |= 1u << p;
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < kRowUnroll; ++q) {  // sources
                    const int j = r0[p] + q;
                    if (j >= r1[p]) continue;
                    const int z = __ldg(A.src + j);
                    const float w = __ldg(A.wt + j);
                    if ((long long)z / SIZE != n_o) {
                        a += w * __ldcg(A.lam + z);
                    } else {  // c <= q < K
                        sm.cw[c][n_i] = w;
                        sm.cz[c][n_i] = (unsigned char)(z - (int)base);
                        ++c;
                    }
                }
                for (int j = r0[p] + kRowUnroll; j < r1[p]; ++j) {  // the rest of a long row
                    const int z = __ldg(A.src + j);
                    const float w = __ldg(A.wt + j);
                    if ((long long)z / SIZE != n_o) {
                        a += w * __ldcg(A.lam + z);
                    } else if (c < K) {
                        sm.cw[c][n_i] = w;
                        sm.cz[c][n_i] = (unsigned char)(z - (int)base);
                        ++c;
                    } else {
                        ovf |= 1u << p;
                    }
                }
            }
            cnt |= (unsigned)c << (4 * p);
            acc[p] = a;
        }
        __syncwarp();
        bool settled = false;
        for (int it = 0; it < kMaxSweeps; ++it) {
            bool moved = false;
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const int n_i = lane + 32 * p;
                float v = acc[p];
                // the in-tile entries in row order: the cached ones, then the rest
                const int c = (int)((cnt >> (4 * p)) & 15u);
#pragma unroll
                for (int k = 0; k < K; ++k)
                    if (k < c) v += sm.cw[k][n_i] * sm.l[sm.cz[k][n_i]];
                if (ovf & (1u << p)) {
                    int seen = 0;
                    if constexpr (FWD) {
                        const long long n_t = base + n_i;
                        for (int k = 0; k < A.nact; ++k) {
                            const float w = __ldg(A.fw + k * I.size_tot + n_t);
                            const int y = __ldg(A.fidx + k * I.size_tot + n_t);
                            if (w != 0.f && y >= 0 && (long long)y / SIZE == n_o && seen++ >= K)
                                v += w * sm.l[y - (int)base];
                        }
                    } else {
                        for (int j = r0[p]; j < r1[p]; ++j) {
                            const int z = __ldg(A.src + j);
                            if ((long long)z / SIZE == n_o && seen++ >= K) v += __ldg(A.wt + j) * sm.l[z - (int)base];
                        }
                    }
                }
                v = v / diag[p];
                __syncwarp();
                if (v != sm.l[n_i]) {
                    sm.l[n_i] = v;
                    moved = true;
                }
                __syncwarp();
            }
            if (!__any_sync(kFull, moved)) {
                settled = true;
                break;
            }
        }
        bool self = !settled;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int n_i = lane + 32 * p;
            const long long n_t = base + n_i;
            const float v = sm.l[n_i];
            __stcg(A.lam + n_t, v);
            const bool changed = fabsf(v - old[p]) > A.atol + A.rtol * fabsf(v);
            if (!changed) continue;
            if constexpr (FWD) {
                for (int j = r0[p]; j < r1[p]; ++j) {  // the points that depend on this one
                    const int ty = __ldg(A.src + j) / SIZE;
                    if (ty == n_o) self = true;
                    else push_tile<false>(S, I, ii, I.tile_base + ty, e);
                }
            } else {
                for (int k = 0; k < A.nact; ++k) {  // the points that depend on this one
                    const float w = __ldg(A.fw + k * I.size_tot + n_t);
                    const int y = __ldg(A.fidx + k * I.size_tot + n_t);
                    if (w == 0.f || y < 0 || (long long)y >= I.size_tot) continue;
                    const int ty = y / SIZE;
                    if (ty == n_o) self = true;
                    else push_tile<false>(S, I, ii, I.tile_base + ty, e);
                }
            }
        }
        __syncwarp();
        if (!settled && lane == 0) push_tile<false>(S, I, ii, t, e);
        (void)self;
    }
};

static inline unsigned nb(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

struct RevLayout {
    WsLayout L;
    size_t rowptr, cursor, src, wt, btot, grand, total;
    long long size_tot;
    int nact, size_i;
};

static bool rev_layout(const agd_instance *a, RevLayout &R, std::vector<Inst> *insts) {
    agd_instance b = *a;
    b.flags = (b.flags | AGD_FLAG_ACTIVATE_ALL) & ~(AGD_FLAG_SOLVER_AGSI | AGD_FLAG_SOLVER_GLOBAL);
    b.trigger = nullptr;
    b.release = nullptr;  // the linear solves keep the two-list schedule
    if (!layout(&b, 1, R.L, insts, /*stencil_cache=*/false)) return false;
    const Inst &I = (*insts)[0];
    R.size_tot = I.size_tot;
    R.size_i = I.size_i;
    R.nact = (a->model == AGD_MODEL_RIEMANN || a->model == AGD_MODEL_RANDER) ? a->ndim * (a->ndim + 1) / 2 : a->ndim;
    size_t off = R.L.total;
    const long long nblk = (R.size_tot + 1 + 1023) / 1024;
    R.rowptr = off; off = align256(off + sizeof(int) * (R.size_tot + 1));
    R.cursor = off; off = align256(off + sizeof(int) * R.size_tot);
    R.src = off; off = align256(off + sizeof(int) * R.nact * R.size_tot);
    R.wt = off; off = align256(off + sizeof(float) * R.nact * R.size_tot);
    R.btot = off; off = align256(off + sizeof(int) * nblk);
    R.grand = off; off = align256(off + sizeof(int));
    R.total = off;
    return true;
}

}  // namespace agd

using namespace agd;

extern "C" {

size_t agd_reverse_workspace_bytes(const agd_instance *inst) {
    if (!inst) return 0;
    RevLayout R;
    std::vector<Inst> v;
    if (!rev_layout(inst, R, &v)) return 0;
    return R.total;
}

}  // extern "C"

namespace agd {

// The transpose of the flow graph, then the linear solve on the tiles.
template <bool FWD>
static int linear_solve(const char *who, const agd_instance *inst, const float *flow_weights,
                        const int32_t *flow_indices, const float *flow_weightsum, const float *rhs, float *sol,
                        float atol, float rtol, void *workspace, size_t workspace_bytes, agd_stats *stats,
                        const agd_launch *launch, cudaStream_t st) {
    char msg[128];
    if (!inst || !flow_weights || !flow_indices || !flow_weightsum || !rhs || !sol || !workspace) {
        snprintf(msg, sizeof(msg), "%s: missing array", who);
        return set_error(AGD_STATUS_INVALID, msg);
    }
    RevLayout R;
    std::vector<Inst> insts;
    if (!rev_layout(inst, R, &insts)) {
        snprintf(msg, sizeof(msg), "%s: bad instance", who);
        return set_error(AGD_STATUS_INVALID, msg);
    }
    if (insts[0].variant < 0) {
        snprintf(msg, sizeof(msg), "%s: tile shape not built", who);
        return set_error(AGD_STATUS_UNSUPPORTED, msg);
    }
    if (workspace_bytes < R.total) {
        snprintf(msg, sizeof(msg), "%s: workspace too small", who);
        return set_error(AGD_STATUS_WORKSPACE, msg);
    }
    char *w = static_cast<char *>(workspace);
    int *rowptr = reinterpret_cast<int *>(w + R.rowptr);
    int *cursor = reinterpret_cast<int *>(w + R.cursor);
    int *src = reinterpret_cast<int *>(w + R.src);
    float *wt = reinterpret_cast<float *>(w + R.wt);
    int *btot = reinterpret_cast<int *>(w + R.btot);
    int *grand = reinterpret_cast<int *>(w + R.grand);
    RevGeom g{R.size_tot, R.nact};
    cudaError_t err = cudaMemsetAsync(cursor, 0, sizeof(int) * R.size_tot, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(sol, 0, sizeof(float) * R.size_tot, st);
    if (err != cudaSuccess) return set_cuda_error("linear solve clear", err);
    // counts (into cursor), exclusive scan into rowptr, then fill
    rev_count_kernel<<<nb(R.size_tot, 256), 256, 0, st>>>(g, flow_weights, flow_indices, cursor);
    const long long n1 = R.size_tot + 1;
    cudaMemsetAsync(rowptr + R.size_tot, 0, sizeof(int), st);
    scan_blocks_kernel<<<nb(n1, 1024), 1024, 0, st>>>(cursor, rowptr, R.size_tot, btot);
    scan_totals_kernel<<<1, 1024, 0, st>>>(btot, (int)nb(n1, 1024), grand);
    scan_add_kernel<<<nb(n1, 1024), 1024, 0, st>>>(rowptr, R.size_tot, btot);
    cudaMemcpyAsync(rowptr + R.size_tot, grand, sizeof(int), cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(cursor, 0, sizeof(int) * R.size_tot, st);
    rev_fill_kernel<<<nb(R.size_tot, 256), 256, 0, st>>>(g, flow_weights, flow_indices, rowptr, cursor, src, wt);
    rev_sort_kernel<<<nb(R.size_tot, 256), 256, 0, st>>>(g, rowptr, src, wt);
    if ((err = cudaGetLastError()) != cudaSuccess) return set_cuda_error("linear solve transpose", err);
    // solve on the tiles
    err = cudaMemcpyAsync(w + R.L.inst, insts.data(), sizeof(Inst), cudaMemcpyHostToDevice, st);
    if (err != cudaSuccess) return set_cuda_error("linear solve descriptor upload", err);
    LinArgs A{rowptr, src, wt, flow_weightsum, rhs, sol, flow_weights, flow_indices, R.nact, atol, rtol};
    if (R.size_i == 256) return run_sched<LinearVisitor<256, FWD>>(R.L, workspace, 1, A, stats, launch, st);
    if (R.size_i == 64) return run_sched<LinearVisitor<64, FWD>>(R.L, workspace, 1, A, stats, launch, st);
    snprintf(msg, sizeof(msg), "%s: tile size not built", who);
    return set_error(AGD_STATUS_UNSUPPORTED, msg);
}

}  // namespace agd

extern "C" {

int agd_reverse(const agd_instance *inst, const float *flow_weights, const int32_t *flow_indices,
                const float *flow_weightsum, const float *sens, float *lam, float atol, float rtol, void *workspace,
                size_t workspace_bytes, agd_stats *stats, const agd_launch *launch, agd_stream_t stream) {
    clear_error();
    return linear_solve<false>("agd_reverse", inst, flow_weights, flow_indices, flow_weightsum, sens, lam, atol, rtol,
                               workspace, workspace_bytes, stats, launch, (cudaStream_t)stream);
}

int agd_forward(const agd_instance *inst, const float *flow_weights, const int32_t *flow_indices,
                const float *flow_weightsum, const float *rhs, float *du, float atol, float rtol, void *workspace,
                size_t workspace_bytes, agd_stats *stats, const agd_launch *launch, agd_stream_t stream) {
    clear_error();
    return linear_solve<true>("agd_forward", inst, flow_weights, flow_indices, flow_weightsum, rhs, du, atol, rtol,
                              workspace, workspace_bytes, stats, launch, (cudaStream_t)stream);
}

}  // extern "C"
