// unet.cu - the learned warm start: a 4-level convolutional U-Net over NHWC
// bf16 activations whose 3x3 convolutions (forward, input gradient and weight
// gradient) are implicit GEMMs on the tcgen05 tensor cores (fp32 accumulators
// in tensor memory), plus the memory-bound layers around them (features,
// pooling, gradient routing, the 1x1 head and its loss, bias gradients, Adam)
// and the two uses of a prediction by the solver: per-tile release epochs and
// warm-start values.  The reference has no learned component; this file has
// no counterpart there.  C ABI: include/agd_warmstart.h.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <cstdint>

#include "../../include/agd_warmstart.h"
#include "agd_internal.h"
#include "umma.cuh"

namespace agd {
namespace unet {

using bf16 = __nv_bfloat16;
constexpr int kBM = 128;           // rows (pixels, or weight rows) per CTA tile
constexpr int kBK = 64;            // K elements per pipeline stage (8 x 16-byte units)
constexpr int kMaxStages = 8;        // operand stages in shared memory (Pipe holds 8 barriers each way)
constexpr int kSmemBudget = 200 * 1024;  // dynamic shared memory of a conv CTA alone on its SM
constexpr int kSmemBudget2 = 104 * 1024; // ... of one of two conv CTAs per SM
constexpr unsigned long long kWaitNs = 2000000000ull;  // bound on every barrier wait

__host__ __device__ inline int kpad_of(int k) { return (k + kBK - 1) / kBK * kBK; }

struct Src {
    const bf16 *p;
    int C;   // channels (multiple of 8)
    int up;  // 1: the tensor is at half resolution, read nearest-upsampled
};

struct GemmArgs {
    int nimg, H, W;  // output (and full-resolution input) shape
    Src s0, s1;      // input channels [0, s0.C) then [s0.C, s0.C + s1.C)
    int cin8;        // (s0.C + s1.C) / 8
    int K8;          // 9 * cin8: 16-byte K units
    int kchunks;     // ceil(K8 / 8)
    int N, BN;       // output channels; channels per CTA tile (multiple of 16, <= 256)
    const bf16 *wmat;  // (N, kpad) bf16, K contiguous
    int kpad;
    const float *bias;
    int relu;
    bf16 *out_bf;
    float *out_f;
    long long M;  // pixels
    int wshift;   // log2(W) when W is a power of two, else -1
    unsigned *err;
};

__device__ __forceinline__ const bf16 *src_ptr(const Src &s, int nb, int y, int x, int H, int W, int ch) {
    const int Hs = H >> s.up, Ws = W >> s.up;
    return s.p + (((long long)nb * Hs + (y >> s.up)) * Ws + (x >> s.up)) * s.C + ch;
}

__device__ __forceinline__ uint32_t tmem_cols(int bn) {
    uint32_t c = 32;
    while (c < (uint32_t)bn) c <<= 1;
    return c;
}

// The convolution GEMMs are persistent and warp-specialised: each CTA loops
// over output tiles; warps 0-3 load operands (cp.async, 16 bytes a lane,
// zero-filled outside the image), warp 4 allocates tensor memory and one of
// its lanes issues the tcgen05 MMAs, warps 5-8 run the epilogue.  Two CTAs
// share an SM where their tensor memory (2 x 2 x BN columns) and shared memory
// allow it: the pipelines' latencies then overlap.  The
// accumulator is double-buffered in tensor memory, so the epilogue of a tile
// overlaps the main loop of the next; operand stages cycle through shared
// memory across tiles.  Every wait is bounded (kWaitNs) and sets *err.
constexpr int kProducers = 128;  // warps 0-3
constexpr int kMmaWarp = kProducers / 32;  // warp 4
constexpr int kEpilogue = 128;   // warps 5-8
constexpr int kPThreads = kProducers + 32 + kEpilogue;  // 288
constexpr int kUnitsPerThread = kBM * 8 / kProducers;  // A units (16 bytes) per producer thread and stage

struct Pipe {
    uint64_t full[8], empty[8], accf[2], acce[2], bready;
    uint32_t taddr;
};

__device__ __forceinline__ void pipe_init(Pipe &P, int stages) {
    for (int s = 0; s < stages; ++s) {
        umma::mbar_init(&P.full[s], kProducers);
        umma::mbar_init(&P.empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
        umma::mbar_init(&P.accf[a], 1);
        umma::mbar_init(&P.acce[a], kEpilogue / 32);
    }
    umma::mbar_init(&P.bready, kProducers);
    umma::fence_mbar_init();
}

// A bounded barrier wait whose result is the same in every lane of the warp
// (false if any lane gave up), so that the warp leaves its loops together.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity, unsigned *err,
                                               unsigned long long timeout_ns) {
    const bool ok = umma::mbar_wait(bar, parity, err, timeout_ns);
    return __all_sync(0xffffffffu, ok);
}

// Before the CTA frees its tensor memory: the MMAs of the last tile are complete
// (its accumulator barrier's phase), also when the epilogue gave up early.
__device__ __forceinline__ void mma_drain(Pipe &P, int ntile_local, unsigned *err) {
    if (ntile_local <= 0) return;
    const int tl = ntile_local - 1;
    mbar_wait_warp(&P.accf[tl & 1], (tl >> 1) & 1, err, kWaitNs);
}

// Ring position of a pipeline stage: index and the parity of its current use.
struct Ring {
    int s = 0;
    uint32_t ph = 0;
    __device__ __forceinline__ void next(int stages) {
        if (++s == stages) {
            s = 0;
            ph ^= 1u;
        }
    }
};

// MMA warp (all lanes wait, lane 0 issues): for each tile, waits for a free
// accumulator, then for each K chunk its stage, issues 4 MMAs of K = 16, frees
// the stage; commits the accumulator.  B: per stage (stationary = false) or one
// resident region of every chunk.
__device__ __forceinline__ void mma_role(Pipe &P, int ntile_local, int nk, uint32_t sbase,
                                         uint32_t stage_bytes, uint32_t a_bytes, int stages, bool stationary,
                                         uint32_t bstat, uint32_t bchunk_bytes, uint32_t idesc, int bn,
                                         unsigned *err) {
    const bool leader = (threadIdx.x & 31) == 0;
    // descriptors advance by the stage size; a K step of 16 is 256 bytes (16 in
    // the descriptor's address field)
    const uint64_t ad0 = umma::smem_desc(sbase, 128u, 1024u);
    const uint64_t bs0 = umma::smem_desc(bstat, 128u, 1024u);
    const uint64_t dstage = stage_bytes >> 4, dab = a_bytes >> 4, dbchunk = bchunk_bytes >> 4;
    Ring R;
    uint64_t ad = ad0;
    bool ok = true;
    if (stationary) ok = mbar_wait_warp(&P.bready, 0, err, kWaitNs);
    for (int tl = 0; tl < ntile_local && ok; ++tl) {
        const int a = tl & 1;
        if (tl >= 2 && !mbar_wait_warp(&P.acce[a], ((tl >> 1) & 1) ^ 1, err, kWaitNs)) break;
        umma::tc_fence_after_sync();
        const uint32_t d = P.taddr + (uint32_t)(a * bn);
        uint64_t bsd = bs0;
        for (int i = 0; i < nk; ++i) {
            if (!mbar_wait_warp(&P.full[R.s], R.ph, err, kWaitNs)) {
                ok = false;
                break;
            }
            umma::fence_proxy_async_smem();  // the producers' cp.async writes before the tensor core reads
            umma::tc_fence_after_sync();
            const uint64_t bd = stationary ? bsd : ad + dab;
            if (leader) {
#pragma unroll
                for (int kk = 0; kk < kBK / 16; ++kk) umma::mma_bf16(d, ad + 16u * kk, bd + 16u * kk, idesc, (i | kk) != 0);
                umma::mma_commit(&P.empty[R.s]);
            }
            __syncwarp();
            bsd += dbchunk;
            ad += dstage;
            R.next(stages);
            if (R.s == 0) ad = ad0;
        }
        if (leader) umma::mma_commit(&P.accf[a]);
        __syncwarp();
    }
    mma_drain(P, ntile_local, err);
}

__device__ __forceinline__ int count_tiles(int total) {
    return total > (int)blockIdx.x ? (total - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
}

// D[m, n] = sum_k A[m, k] B[n, k]: A the implicit im2col of the input (m a
// pixel, k = tap * cin + ci, tap = 3 (dy + 1) + (dx + 1), zero outside the
// image), B the weight matrix.  Epilogue: + bias, ReLU, bf16 or fp32 NHWC.
// Shared memory per stage: A 128 x 64 and B BN x 64 bf16 in the no-swizzle
// K-major core-matrix layout (16-byte unit u at byte 16 u, u = (row / 8) * 64 +
// kunit * 8 + row % 8), which makes every producer lane's unit a single cp.async.
// With one channel tile and small weights, B stays resident for the whole launch.
struct GemmLaunch {
    int stages, stationary, mtiles, ntiles;
};

__global__ void __launch_bounds__(kPThreads, 2) conv_gemm_kernel(GemmArgs g, GemmLaunch gl) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ Pipe P;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ncols = tmem_cols(2 * g.BN);
    const uint32_t a_bytes = kBM * kBK * 2, bchunk = (uint32_t)g.BN * kBK * 2;
    const uint32_t stage_bytes = a_bytes + (gl.stationary ? 0u : bchunk);
    const uint32_t sbase = umma::smem_u32(smem);
    const uint32_t bstat = sbase + gl.stages * stage_bytes;
    const int total = gl.mtiles * gl.ntiles;
    const int ntl = count_tiles(total);

    if (warp == kMmaWarp) {
        umma::tmem_alloc(&P.taddr, ncols);
        umma::tmem_relinquish();
    }
    if (tid == 0) pipe_init(P, gl.stages);
    umma::tc_fence_before_sync();
    __syncthreads();
    umma::tc_fence_after_sync();

    if (warp < kMmaWarp) {
        // ---------------------------------------------------------- producer
        if (gl.stationary) {  // every chunk of B once
            const int units = g.kchunks * g.BN * 8;
            for (int v = tid; v < units; v += kProducers) {
                const int i = v / (g.BN * 8), u = v - i * (g.BN * 8);
                const int n = ((u >> 6) << 3) + (u & 7);
                const int kk = i * 8 + ((u >> 3) & 7);
                const bool ok = n < g.N && kk < g.K8;
                const void *src = ok ? (const void *)(g.wmat + (long long)n * g.kpad + kk * 8) : (const void *)g.wmat;
                umma::cp_async16(bstat + i * bchunk + 16u * u, src, ok ? 16u : 0u);
            }
            umma::cp_async_mbar_arrive(&P.bready);
        }
        // A: rows 8 ((tid >> 6) + (kProducers / 64) j) + (tid & 7), j < kUnitsPerThread, K unit c = (tid >> 3) & 7
        // of each chunk.  Per tile: each row's pixel address in both inputs and
        // its mask of taps inside the image (bits 0-8) with the pixel's row and
        // column parities (bits 9, 10: the offsets of an upsampled input).
        const int c = (tid >> 3) & 7;
        const int C0 = g.s0.C, C1 = g.s1.C, W0s = g.W >> g.s0.up, W1s = g.W >> g.s1.up;
        Ring R;
        bool wrapped = false, alive = true;
        for (int tl = 0; tl < ntl && alive; ++tl) {
            const int t = blockIdx.x + tl * gridDim.x;
            const int mt = t % gl.mtiles, nt = t / gl.mtiles;
            const long long m0 = (long long)mt * kBM;
            const int n0 = nt * g.BN;
            const bf16 *b0[kUnitsPerThread], *b1[kUnitsPerThread];
            unsigned vm[kUnitsPerThread];
            // image of the tile's first row; rows beyond it (a tile straddling
            // two images) step to the next image below
            const int hw = g.H * g.W;
            const int nb0 = (int)(m0 / hw);
            const int r0 = (int)(m0 - (long long)nb0 * hw);
#pragma unroll
            for (int j = 0; j < kUnitsPerThread; ++j) {
                const int row = 8 * ((tid >> 6) + (kProducers / 64) * j) + (tid & 7);
                vm[j] = 0u;
                b0[j] = b1[j] = g.s0.p;
                if (m0 + row < g.M) {
                    int r = r0 + row, nb = nb0;
                    while (r >= hw) {  // at most kBM / hw + 1 steps
                        r -= hw;
                        ++nb;
                    }
                    const int y = g.wshift >= 0 ? r >> g.wshift : r / g.W;
                    const int x = r - y * g.W;
                    b0[j] = src_ptr(g.s0, nb, y, x, g.H, g.W, 0);
                    if (g.s1.p) b1[j] = src_ptr(g.s1, nb, y, x, g.H, g.W, 0);
                    unsigned mk = 0u;
#pragma unroll
                    for (int tap = 0; tap < 9; ++tap) {
                        const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
                        mk |= (yy >= 0 && yy < g.H && xx >= 0 && xx < g.W) ? (1u << tap) : 0u;
                    }
                    vm[j] = mk | ((unsigned)(y & 1) << 9) | ((unsigned)(x & 1) << 10);
                }
            }
            int tap = c / g.cin8, ci8 = c - (c / g.cin8) * g.cin8;  // of unit c of chunk 0
            for (int i = 0; i < g.kchunks; ++i) {
                if (wrapped && !mbar_wait_warp(&P.empty[R.s], R.ph ^ 1u, g.err, kWaitNs)) {
                    alive = false;
                    break;
                }
                const uint32_t sa = sbase + R.s * stage_bytes, sb = sa + a_bytes;
                const bool kin = tap < 9;
                const int dy = tap / 3 - 1, dx = tap - 3 * (tap / 3) - 1;
                const bool first = ci8 * 8 < C0;
                const int ch = first ? ci8 * 8 : ci8 * 8 - C0;
                const int up = first ? g.s0.up : g.s1.up;
                const int Cs = first ? C0 : C1, Ws = first ? W0s : W1s;
                const long long offp = (long long)(dy * Ws + dx) * Cs + ch;  // same-resolution input
#pragma unroll
                for (int j = 0; j < kUnitsPerThread; ++j) {
                    const int u = tid + kProducers * j;
                    const bool ok = kin && ((vm[j] >> tap) & 1u);
                    long long off = offp;
                    if (up) {
                        const int ey = (int)((vm[j] >> 9) & 1u) + dy, ex = (int)((vm[j] >> 10) & 1u) + dx;
                        off = (long long)((ey >> 1) * Ws + (ex >> 1)) * Cs + ch;
                    }
                    const void *src = ok ? (const void *)((first ? b0[j] : b1[j]) + off) : (const void *)g.wmat;
                    umma::cp_async16(sa + 16u * u, src, ok ? 16u : 0u);
                }
                if (!gl.stationary) {
                    for (int u = tid; u < g.BN * 8; u += kProducers) {
                        const int n = n0 + ((u >> 6) << 3) + (u & 7);
                        const int kk = i * 8 + ((u >> 3) & 7);
                        const bool ok = n < g.N && kk < g.K8;
                        const void *src =
                            ok ? (const void *)(g.wmat + (long long)n * g.kpad + kk * 8) : (const void *)g.wmat;
                        umma::cp_async16(sb + 16u * u, src, ok ? 16u : 0u);
                    }
                }
                umma::cp_async_mbar_arrive(&P.full[R.s]);
                R.next(gl.stages);
                wrapped = wrapped || R.s == 0;
                // unit c of the next chunk: 8 units further along K
                ci8 += 8;
                while (ci8 >= g.cin8 && tap < 9) {
                    ci8 -= g.cin8;
                    ++tap;
                }
            }
        }
    } else if (warp == kMmaWarp) {
        {
            mma_role(P, ntl, g.kchunks, sbase, stage_bytes, a_bytes, gl.stages, gl.stationary != 0, bstat, bchunk,
                     umma::idesc_bf16(kBM, g.BN, 0, 0), g.BN, g.err);
        }
    } else {
        // ---------------------------------------------------------- epilogue
        const int ew = warp & 3;  // TMEM lane quarter of this warp
        for (int tl = 0; tl < ntl; ++tl) {
            const int a = tl & 1;
            const bool ok = mbar_wait_warp(&P.accf[a], (tl >> 1) & 1, g.err, kWaitNs);
            umma::tc_fence_after_sync();
            if (!ok) break;
            const int t = blockIdx.x + tl * gridDim.x;
            const int mt = t % gl.mtiles, nt = t / gl.mtiles;
            const long long m = (long long)mt * kBM + 32 * ew + lane;
            for (int c0 = 0; c0 < g.BN; c0 += 16) {
                uint32_t r[16];
                umma::tmem_ld16(P.taddr + ((uint32_t)(32 * ew) << 16) + (uint32_t)(a * g.BN + c0), r);
                umma::tmem_ld_wait();
                const int nc = nt * g.BN + c0;
                if (m >= g.M || nc >= g.N) continue;
                float v[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    v[q] = __uint_as_float(r[q]);
                    if (g.bias) v[q] += __ldg(g.bias + nc + q);
                    if (g.relu) v[q] = fmaxf(v[q], 0.f);
                }
                if (g.out_bf) {
                    uint4 w[2];
                    uint32_t *wp = reinterpret_cast<uint32_t *>(w);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                        wp[q] = *reinterpret_cast<uint32_t *>(&h);
                    }
                    uint4 *dst = reinterpret_cast<uint4 *>(g.out_bf + m * g.N + nc);
                    dst[0] = w[0];
                    dst[1] = w[1];
                } else {
                    float4 *dst = reinterpret_cast<float4 *>(g.out_f + m * g.N + nc);
#pragma unroll
                    for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                }
            }
            umma::tc_fence_before_sync();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_u32(&P.acce[a])) : "memory");
        }
    }
    umma::cp_async_wait_all();
    umma::tc_fence_before_sync();
    __syncthreads();
    if (warp == kMmaWarp) {
        umma::tc_fence_after_sync();
        umma::tmem_dealloc(P.taddr, ncols);
    }
}

// --------------------------------------------------------- TMA-fed forward
// The same GEMM with both operands moved by bulk tensor copies (TMA) into
// swizzled K-major tiles, for inputs whose channel counts are multiples of 32
// at the output's resolution, images of W | 128 columns and 128 | H W pixels:
// a tile is 128 / W whole rows of one image.  A K chunk is (tap, input,
// block of CB = 64 channels, or 32 for a 32-channel input): the A tile is the
// box (CB channels, W columns, 128 / W rows) of the input at (channel block,
// dx, y0 + dy, image), zero outside the image by the copy's out-of-bounds
// fill, in 128-byte (64-byte) swizzled rows; the B tile the box (CB, BN) of
// the weight matrix at (tap cin + channel offset, n0).  One producer lane
// issues both copies per stage against one mbarrier transaction count, so
// the operands bypass the per-lane L1 path.
struct TmaArgs {
    int H, W, R;       // rows of the output, columns, rows per tile (128 / W)
    int C0, C1;        // input channels
    int cb0, cb1;      // channel block of each input (64 or 32)
    int cin, N, BN, kchunks;
    int spc;           // K chunks per pipeline stage (each in its own slot)
    int rowmax;        // bytes of the widest tile row (2 x the largest channel block)
    const float *bias;
    int relu;
    bf16 *out_bf;
    float *out_f;
    long long M;
    int mtiles, ntiles, stages;
    unsigned *err;
};

// K chunk i -> (input s, channel offset c in that input, tap); the order is
// tap-major, then the inputs' channel blocks.
__device__ __forceinline__ void tma_chunk(const TmaArgs &g, int i, int &s, int &c, int &tap) {
    const int per = g.C0 / g.cb0 + (g.C1 ? g.C1 / g.cb1 : 0);
    tap = i / per;
    const int j = i - tap * per;
    const int n0 = g.C0 / g.cb0;
    if (j < n0) {
        s = 0;
        c = j * g.cb0;
    } else {
        s = 1;
        c = (j - n0) * g.cb1;
    }
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(umma::smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(umma::smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// K-major swizzled descriptor: rows of `row` bytes (128: 128-byte swizzle,
// 64: 64-byte swizzle), 8-row atoms of 8 row bytes.
__device__ __forceinline__ uint64_t swz_desc(uint32_t saddr, int row) {
    const uint64_t layout = row == 128 ? 2ull : 4ull;
    return (uint64_t)((saddr >> 4) & 0x3fffu) | (1ull << 16) | ((uint64_t)(((8u * row) >> 4) & 0x3fffu) << 32) |
           (1ull << 46) | (layout << 61);
}

__global__ void __launch_bounds__(kPThreads, 2)
    conv_tma_kernel(TmaArgs g, const __grid_constant__ CUtensorMap xa0, const __grid_constant__ CUtensorMap xa1,
                    const __grid_constant__ CUtensorMap wb64, const __grid_constant__ CUtensorMap wb32) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ Pipe P;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ncols = tmem_cols(2 * g.BN);
    const uint32_t a_bytes = kBM * g.rowmax, b_bytes = (uint32_t)g.BN * g.rowmax;  // a slot: the widest block
    const uint32_t slot_bytes = a_bytes + b_bytes, stage_bytes = slot_bytes * g.spc;
    const uint32_t sbase = (umma::smem_u32(smem) + 1023u) & ~1023u;  // swizzle atoms on 1024-byte boundaries
    const int ntl = count_tiles(g.mtiles * g.ntiles);
    const int nstage = (g.kchunks + g.spc - 1) / g.spc;  // stages per tile

    if (warp == kMmaWarp) {
        umma::tmem_alloc(&P.taddr, ncols);
        umma::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < g.stages; ++s) {
            umma::mbar_init(&P.full[s], 1);
            umma::mbar_init(&P.empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            umma::mbar_init(&P.accf[a], 1);
            umma::mbar_init(&P.acce[a], kEpilogue / 32);
        }
        umma::fence_mbar_init();
    }
    umma::tc_fence_before_sync();
    __syncthreads();
    umma::tc_fence_after_sync();

    if (warp == 0) {
        // ---------------------------------------------- producer (one lane)
        Ring R;
        bool wrapped = false, alive = true;
        for (int tl = 0; tl < ntl && alive; ++tl) {
            const int t = blockIdx.x + tl * gridDim.x;
            const int mt = t % g.mtiles, nt = t / g.mtiles;
            const long long m0 = (long long)mt * kBM;
            const int nimg = (int)(m0 / ((long long)g.H * g.W));
            const int y0 = (int)((m0 - (long long)nimg * g.H * g.W) / g.W);
            for (int i0 = 0; i0 < nstage; ++i0) {
                if (wrapped && !mbar_wait_warp(&P.empty[R.s], R.ph ^ 1u, g.err, kWaitNs)) {
                    alive = false;
                    break;
                }
                if (lane == 0) {
                    const int i1 = min(g.kchunks, (i0 + 1) * g.spc);
                    uint32_t tx = 0;
                    for (int i = i0 * g.spc; i < i1; ++i) {
                        int s, c, tap;
                        tma_chunk(g, i, s, c, tap);
                        tx += (uint32_t)(kBM + g.BN) * (s ? g.cb1 : g.cb0) * 2;
                    }
                    mbar_expect_tx(&P.full[R.s], tx);
                    for (int i = i0 * g.spc; i < i1; ++i) {
                        int s, c, tap;
                        tma_chunk(g, i, s, c, tap);
                        const int cb = s ? g.cb1 : g.cb0;
                        const uint32_t sa = sbase + R.s * stage_bytes + (i - i0 * g.spc) * slot_bytes, sb = sa + a_bytes;
                        tma_load_4d(sa, s ? &xa1 : &xa0, c, tap % 3 - 1, y0 + tap / 3 - 1, nimg, &P.full[R.s]);
                        tma_load_2d(sb, cb == 64 ? &wb64 : &wb32, tap * g.cin + (s ? g.C0 : 0) + c, nt * g.BN,
                                    &P.full[R.s]);
                    }
                }
                __syncwarp();
                R.next(g.stages);
                wrapped = wrapped || R.s == 0;
            }
        }
    } else if (warp == kMmaWarp) {
        // ---------------------------------------------- MMA (lane 0 issues)
        const bool leader = lane == 0;
        const uint32_t idesc = umma::idesc_bf16(kBM, g.BN, 0, 0);
        Ring R;
        bool ok = true;
        for (int tl = 0; tl < ntl && ok; ++tl) {
            const int a = tl & 1;
            if (tl >= 2 && !mbar_wait_warp(&P.acce[a], ((tl >> 1) & 1) ^ 1, g.err, kWaitNs)) break;
            umma::tc_fence_after_sync();
            const uint32_t d = P.taddr + (uint32_t)(a * g.BN);
            for (int i0 = 0; i0 < nstage; ++i0) {
                if (!mbar_wait_warp(&P.full[R.s], R.ph, g.err, kWaitNs)) {
                    ok = false;
                    break;
                }
                umma::tc_fence_after_sync();
                if (leader) {
                    const int i1 = min(g.kchunks, (i0 + 1) * g.spc);
                    for (int i = i0 * g.spc; i < i1; ++i) {
                        int s, c, tap;
                        tma_chunk(g, i, s, c, tap);
                        const int row = 2 * (s ? g.cb1 : g.cb0);  // bytes of a tile row
                        const uint32_t sa = sbase + R.s * stage_bytes + (i - i0 * g.spc) * slot_bytes, sb = sa + a_bytes;
                        const uint64_t ad = swz_desc(sa, row), bd = swz_desc(sb, row);
                        for (int kk = 0; kk < row / 32; ++kk)  // K = 16 per MMA: 32 bytes of a row
                            umma::mma_bf16(d, ad + 2u * kk, bd + 2u * kk, idesc, (i | kk) != 0);
                    }
                    umma::mma_commit(&P.empty[R.s]);
                }
                __syncwarp();
                R.next(g.stages);
            }
            if (leader) umma::mma_commit(&P.accf[a]);
            __syncwarp();
        }
        mma_drain(P, ntl, g.err);
    } else if (warp > kMmaWarp) {
        // ---------------------------------------------------------- epilogue
        const int ew = warp & 3;
        for (int tl = 0; tl < ntl; ++tl) {
            const int a = tl & 1;
            const bool ok = mbar_wait_warp(&P.accf[a], (tl >> 1) & 1, g.err, kWaitNs);
            umma::tc_fence_after_sync();
            if (!ok) break;
            const int t = blockIdx.x + tl * gridDim.x;
            const int mt = t % g.mtiles, nt = t / g.mtiles;
            const long long m = (long long)mt * kBM + 32 * ew + lane;
            for (int c0 = 0; c0 < g.BN; c0 += 16) {
                uint32_t r[16];
                umma::tmem_ld16(P.taddr + ((uint32_t)(32 * ew) << 16) + (uint32_t)(a * g.BN + c0), r);
                umma::tmem_ld_wait();
                const int nc = nt * g.BN + c0;
                if (m >= g.M || nc >= g.N) continue;
                float v[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    v[q] = __uint_as_float(r[q]);
                    if (g.bias) v[q] += __ldg(g.bias + nc + q);
                    if (g.relu) v[q] = fmaxf(v[q], 0.f);
                }
                if (g.out_bf) {
                    uint4 w[2];
                    uint32_t *wp = reinterpret_cast<uint32_t *>(w);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                        wp[q] = *reinterpret_cast<uint32_t *>(&h);
                    }
                    uint4 *dst = reinterpret_cast<uint4 *>(g.out_bf + m * g.N + nc);
                    dst[0] = w[0];
                    dst[1] = w[1];
                } else {
                    float4 *dst = reinterpret_cast<float4 *>(g.out_f + m * g.N + nc);
#pragma unroll
                    for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                }
            }
            umma::tc_fence_before_sync();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_u32(&P.acce[a])) : "memory");
        }
    }
    umma::tc_fence_before_sync();
    __syncthreads();
    if (warp == kMmaWarp) {
        umma::tc_fence_after_sync();
        umma::tmem_dealloc(P.taddr, ncols);
    }
}

// Weight gradient: dW[n, r] += sum_p dZ[p, n] X[p + tap(r), ci(r)], r = tap *
// cin + ci.  GEMM with M = r (128 per tile), N = n, K = pixels (64 per stage,
// split over `splits` work items): both operands MN-major (8 consecutive
// channels of one pixel per 16-byte unit, as they lie in NHWC memory).  Shared
// layout: unit (group g of 8 rows, pixel k) at byte 16 (g * 64 + k).  Work
// item t: row tile t % mtiles, channel tile (t / mtiles) % ntiles, split
// t / (mtiles ntiles); its partial sums go to dw by atomic adds.
struct WgradArgs {
    int nimg, H, W;
    Src s0, s1;
    int cin8, K8;
    const bf16 *dz;  // (M, N) bf16
    int N, BN;
    float *dw;       // (N, kpad) fp32, accumulated
    int kpad;
    long long M;
    int nchunks, chunks_per_split;
    int mtiles, ntiles, splits, stages;
    int wshift;  // log2(W) when W is a power of two, else -1
    unsigned *err;
};

__global__ void __launch_bounds__(kPThreads, 2) conv_wgrad_kernel(WgradArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ Pipe P;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ncols = tmem_cols(2 * g.BN);
    const uint32_t a_bytes = kBM * kBK * 2, b_bytes = (uint32_t)g.BN * kBK * 2;
    const uint32_t stage_bytes = a_bytes + b_bytes;
    const uint32_t sbase = umma::smem_u32(smem);
    const int total = g.mtiles * g.ntiles * g.splits;
    const int ntl = count_tiles(total);
    // every split has chunks_per_split chunks except possibly the last; the MMA
    // and the producers agree on each item's count through item_chunks()
    auto item_chunks = [&](int t) {
        const int sp = t / (g.mtiles * g.ntiles);
        return min(g.nchunks, (sp + 1) * g.chunks_per_split) - sp * g.chunks_per_split;
    };

    if (warp == kMmaWarp) {
        umma::tmem_alloc(&P.taddr, ncols);
        umma::tmem_relinquish();
    }
    if (tid == 0) pipe_init(P, g.stages);
    umma::tc_fence_before_sync();
    __syncthreads();
    umma::tc_fence_after_sync();

    if (warp < kMmaWarp) {
        const int pk = tid & 63;
        Ring R;
        bool wrapped = false, alive = true;
        for (int tl = 0; tl < ntl && alive; ++tl) {
            const int t = blockIdx.x + tl * gridDim.x;
            const int mt = t % g.mtiles, nt = (t / g.mtiles) % g.ntiles, sp = t / (g.mtiles * g.ntiles);
            const int n0 = nt * g.BN;
            // the weight-row groups of this thread, (tid >> 6) + (kProducers / 64) j: tap, source, channel
            int gtap[kUnitsPerThread], gch[kUnitsPerThread], gsrc[kUnitsPerThread];
#pragma unroll
            for (int j = 0; j < kUnitsPerThread; ++j) {
                const int kk8 = mt * 16 + (tid >> 6) + (kProducers / 64) * j;
                if (kk8 < g.K8) {
                    const int tap = kk8 / g.cin8, ci8 = kk8 - (kk8 / g.cin8) * g.cin8;
                    gtap[j] = tap;
                    gsrc[j] = ci8 * 8 < g.s0.C ? 0 : 1;
                    gch[j] = gsrc[j] ? ci8 * 8 - g.s0.C : ci8 * 8;
                } else {
                    gsrc[j] = -1;
                    gtap[j] = gch[j] = 0;
                }
            }
            const int nk = item_chunks(t);
            const int hw = g.H * g.W;
            // this thread's pixel of the item's first chunk; it advances by kBK a chunk
            long long p = (long long)sp * g.chunks_per_split * kBK + pk;
            int pnb = (int)(p / hw), pr = (int)(p - (long long)pnb * hw);
            for (int i = 0; i < nk; ++i, p += kBK) {
                if (wrapped && !mbar_wait_warp(&P.empty[R.s], R.ph ^ 1u, g.err, kWaitNs)) {
                    alive = false;
                    break;
                }
                const uint32_t sa = sbase + R.s * stage_bytes, sb = sa + a_bytes;
                int nb = -1, y = 0, x = 0;
                if (p < g.M) {
                    nb = pnb;
                    y = g.wshift >= 0 ? pr >> g.wshift : pr / g.W;
                    x = pr - y * g.W;
                }
                pr += kBK;
                while (pr >= hw) {
                    pr -= hw;
                    ++pnb;
                }
#pragma unroll
                for (int j = 0; j < kUnitsPerThread; ++j) {
                    const int u = tid + kProducers * j;
                    const int yy = y + gtap[j] / 3 - 1, xx = x + gtap[j] % 3 - 1;
                    const bool ok = nb >= 0 && gsrc[j] >= 0 && yy >= 0 && yy < g.H && xx >= 0 && xx < g.W;
                    const Src &S = gsrc[j] == 1 ? g.s1 : g.s0;
                    const void *src = ok ? (const void *)src_ptr(S, nb, yy, xx, g.H, g.W, gch[j]) : (const void *)g.dz;
                    umma::cp_async16(sa + 16u * u, src, ok ? 16u : 0u);
                }
                const bf16 *dzp = g.dz + p * g.N;
                for (int u = tid; u < g.BN * 8; u += kProducers) {
                    const int n = n0 + ((u >> 6) << 3);
                    const bool ok = nb >= 0 && n < g.N;
                    const void *src = ok ? (const void *)(dzp + n) : (const void *)g.dz;
                    umma::cp_async16(sb + 16u * u, src, ok ? 16u : 0u);
                }
                umma::cp_async_mbar_arrive(&P.full[R.s]);
                R.next(g.stages);
                wrapped = wrapped || R.s == 0;
            }
        }
    } else if (warp == kMmaWarp) {
        {
            // all lanes wait, lane 0 issues; per-item chunk counts differ only
            // for the last split, so the loop is written out here
            const bool leader = lane == 0;
            const uint32_t idesc = umma::idesc_bf16(kBM, g.BN, 1, 1);
            const uint64_t ad0 = umma::smem_desc(sbase, 128u, 1024u);
            const uint64_t dstage = stage_bytes >> 4, dab = a_bytes >> 4;
            Ring R;
            uint64_t ad = ad0;
            for (int tl = 0; tl < ntl; ++tl) {
                const int a = tl & 1;
                if (tl >= 2 && !mbar_wait_warp(&P.acce[a], ((tl >> 1) & 1) ^ 1, g.err, kWaitNs)) break;
                umma::tc_fence_after_sync();
                const uint32_t d = P.taddr + (uint32_t)(a * g.BN);
                const int nk = item_chunks(blockIdx.x + tl * gridDim.x);
                bool ok = true;
                for (int i = 0; i < nk; ++i) {
                    if (!mbar_wait_warp(&P.full[R.s], R.ph, g.err, kWaitNs)) {
                        ok = false;
                        break;
                    }
                    umma::fence_proxy_async_smem();
                    umma::tc_fence_after_sync();
                    if (leader) {
#pragma unroll
                        for (int kk = 0; kk < kBK / 16; ++kk)
                            umma::mma_bf16(d, ad + 16u * kk, ad + dab + 16u * kk, idesc, (i | kk) != 0);
                        umma::mma_commit(&P.empty[R.s]);
                    }
                    __syncwarp();
                    ad += dstage;
                    R.next(g.stages);
                    if (R.s == 0) ad = ad0;
                }
                if (leader) umma::mma_commit(&P.accf[a]);
                __syncwarp();
                if (!ok) break;
            }
            mma_drain(P, ntl, g.err);
        }
    } else {
        const int ew = warp & 3;
        for (int tl = 0; tl < ntl; ++tl) {
            const int a = tl & 1;
            const bool ok = mbar_wait_warp(&P.accf[a], (tl >> 1) & 1, g.err, kWaitNs);
            umma::tc_fence_after_sync();
            if (!ok) break;
            const int t = blockIdx.x + tl * gridDim.x;
            const int mt = t % g.mtiles, nt = (t / g.mtiles) % g.ntiles;
            const int r = mt * kBM + 32 * ew + lane;  // weight row (tap, ci)
            const bool rin = r < g.K8 * 8;
            for (int c0 = 0; c0 < g.BN; c0 += 16) {
                uint32_t v[16];
                umma::tmem_ld16(P.taddr + ((uint32_t)(32 * ew) << 16) + (uint32_t)(a * g.BN + c0), v);
                umma::tmem_ld_wait();
                if (!rin) continue;
#pragma unroll
                for (int qq = 0; qq < 16; ++qq) {
                    const int n = nt * g.BN + c0 + qq;
                    if (n < g.N) atomicAdd(g.dw + (long long)n * g.kpad + r, __uint_as_float(v[qq]));
                }
            }
            umma::tc_fence_before_sync();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_u32(&P.acce[a])) : "memory");
        }
    }
    umma::cp_async_wait_all();
    umma::tc_fence_before_sync();
    __syncthreads();
    if (warp == kMmaWarp) {
        umma::tc_fence_after_sync();
        umma::tmem_dealloc(P.taddr, ncols);
    }
}

// ------------------------------------------------------- memory-bound layers
// Input features of Riemann2 problems: per output pixel (a 4x4 block of the
// grid), the block mean of the metric (a = (m00 + m11) / 2, b = (m00 - m11) / 2,
// c = m10): log(a) / 4, b / a, c / a; the Euclidean distance d from the block
// centre to the nearest seed (domain units), log(d + 2 h) / 4, 1, 0, 0.
// dref = d + 2 h, the scale of the predicted arrival time.
__global__ void features_kernel(const float *metric, const float *seeds, int nseeds, int n, int H, int W, float h,
                                bf16 *x0, float *dref) {
    const int Ho = H / 4, Wo = W / 4;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * Ho * Wo) return;
    const int b = (int)(idx / (Ho * Wo));
    const int r = (int)(idx - (long long)b * Ho * Wo);
    const int oy = r / Wo, ox = r - (r / Wo) * Wo;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    for (int dy = 0; dy < 4; ++dy)
        for (int dx = 0; dx < 4; ++dx) {
            const float *m = metric + (((long long)b * H + 4 * oy + dy) * W + 4 * ox + dx) * 3;
            s0 += __ldg(m);
            s1 += __ldg(m + 1);
            s2 += __ldg(m + 2);
        }
    s0 *= 1.f / 16;
    s1 *= 1.f / 16;
    s2 *= 1.f / 16;
    const float a = 0.5f * (s0 + s2), bb = 0.5f * (s0 - s2);
    // block centre in domain units: index (4 oy + 1.5) at cell centres (i + 0.5) h
    const float cy = (4.f * oy + 2.f) * h, cx = (4.f * ox + 2.f) * h;
    float d2 = 1e30f;
    for (int k = 0; k < nseeds; ++k) {
        const float sy = __ldg(seeds + ((long long)b * nseeds + k) * 2), sx = __ldg(seeds + ((long long)b * nseeds + k) * 2 + 1);
        d2 = fminf(d2, (sy - cy) * (sy - cy) + (sx - cx) * (sx - cx));
    }
    const float d = sqrtf(d2);
    const float f[8] = {0.25f * logf(a), bb / a, s1 / a, d, 0.25f * logf(d + 2.f * h), 1.f, 0.f, 0.f};
    uint4 w;
    uint32_t *wp = reinterpret_cast<uint32_t *>(&w);
    for (int q = 0; q < 4; ++q) {
        __nv_bfloat162 v = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
        wp[q] = *reinterpret_cast<uint32_t *>(&v);
    }
    reinterpret_cast<uint4 *>(x0)[idx] = w;
    dref[idx] = d + 2.f * h;
}

// Training target: log of the 4x4 block mean of the arrival times over dref.
__global__ void target_kernel(const float *values, int n, int H, int W, const float *dref, float *target) {
    const int Ho = H / 4, Wo = W / 4;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * Ho * Wo) return;
    const int b = (int)(idx / (Ho * Wo));
    const int r = (int)(idx - (long long)b * Ho * Wo);
    const int oy = r / Wo, ox = r - (r / Wo) * Wo;
    float s = 0.f;
    for (int dy = 0; dy < 4; ++dy)
        for (int dx = 0; dx < 4; ++dx) s += __ldg(values + ((long long)b * H + 4 * oy + dy) * W + 4 * ox + dx);
    s *= 1.f / 16;
    target[idx] = isfinite(s) && s > 0.f ? logf(s / dref[idx]) : __int_as_float(0x7fc00000);
}

// 2x2 average pooling, NHWC bf16, 8 channels per thread.
__global__ void avgpool_kernel(const bf16 *x, int n, int H, int W, int C, bf16 *y) {
    const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * Ho * Wo * C8) return;
    const int c8 = (int)(idx % C8);
    const long long p = idx / C8;
    const int b = (int)(p / (Ho * Wo));
    const int r = (int)(p - (long long)b * Ho * Wo);
    const int oy = r / Wo, ox = r - (r / Wo) * Wo;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
            const uint4 v = *reinterpret_cast<const uint4 *>(x + (((long long)b * H + 2 * oy + dy) * W + 2 * ox + dx) * C + c8 * 8);
            const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
            for (int q = 0; q < 4; ++q) {
                const float2 f = __bfloat1622float2(h[q]);
                acc[2 * q] += f.x;
                acc[2 * q + 1] += f.y;
            }
        }
    uint4 w;
    __nv_bfloat162 *wh = reinterpret_cast<__nv_bfloat162 *>(&w);
    for (int q = 0; q < 4; ++q) wh[q] = __floats2bfloat162_rn(0.25f * acc[2 * q], 0.25f * acc[2 * q + 1]);
    *reinterpret_cast<uint4 *>(y + p * C + c8 * 8) = w;
}

// Nearest 2x upsampling, NHWC bf16 (n, H, W, C) -> (n, 2H, 2W, C), 8 channels per thread.
__global__ void upsample_kernel(const bf16 *x, int n, int H, int W, int C, bf16 *y) {
    const int C8 = C / 8;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * 4 * H * W * C8) return;
    const int c8 = (int)(idx % C8);
    const long long p = idx / C8;  // output pixel
    const int b = (int)(p / (4LL * H * W));
    const int r = (int)(p - (long long)b * 4 * H * W);
    const int oy = r / (2 * W), ox = r - (r / (2 * W)) * (2 * W);
    *reinterpret_cast<uint4 *>(y + p * C + c8 * 8) =
        *reinterpret_cast<const uint4 *>(x + (((long long)b * H + oy / 2) * W + ox / 2) * C + c8 * 8);
}

// Backward routing into a layer output Y (n, H, W, C): the gradient of Y is the
// sum of up to two terms, each read from an fp32 NHWC buffer of Cb channels at
// channel offset `off`: SAME (same resolution), POOL (the input gradient of a
// 2x2 average pool of Y: the buffer at half resolution, times 1/4) or UPSUM
// (the input gradient of a nearest 2x upsampling of Y: the sum of the 2x2
// buffer pixels at double resolution); times the ReLU mask Y > 0, to bf16.
struct RouteTerm {
    const float *p;
    int mode;  // 0 none, 1 SAME, 2 POOL, 3 UPSUM
    int Cb, off;
};

__global__ void route_kernel(int n, int H, int W, int C, const bf16 *y, RouteTerm t0, RouteTerm t1, bf16 *dz) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * H * W * C) return;
    const int c = (int)(idx % C);
    const long long p = idx / C;
    const int b = (int)(p / ((long long)H * W));
    const int r = (int)(p - (long long)b * H * W);
    const int py = r / W, px = r - (r / W) * W;
    float g = 0.f;
    const RouteTerm ts[2] = {t0, t1};
    for (int k = 0; k < 2; ++k) {
        const RouteTerm &t = ts[k];
        if (t.mode == 1) {
            g += t.p[p * t.Cb + t.off + c];
        } else if (t.mode == 2) {
            g += 0.25f * t.p[(((long long)b * (H / 2) + py / 2) * (W / 2) + px / 2) * t.Cb + t.off + c];
        } else if (t.mode == 3) {
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx)
                    g += t.p[(((long long)b * (2 * H) + 2 * py + dy) * (2 * W) + 2 * px + dx) * t.Cb + t.off + c];
        }
    }
    if (y && !(__bfloat162float(y[idx]) > 0.f)) g = 0.f;
    dz[idx] = __float2bfloat16_rn(g);
}

// Bias gradient: db[c] += sum over pixels of dz[p, c].
__global__ void bias_grad_kernel(const bf16 *dz, long long M, int C, float *db) {
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    const int j = threadIdx.x / C;
    if (j >= lanes) return;
    float s = 0.f;
    for (long long p = (long long)blockIdx.x * lanes + j; p < M; p += (long long)gridDim.x * lanes)
        s += __bfloat162float(dz[p * C + c]);
    atomicAdd(db + c, s);
}

// 1x1 head: r[p] = sum_c y[p, c] w[c] + b (C = 32).
__global__ void head_forward_kernel(const bf16 *y, long long M, const float *w, const float *b, float *r) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    float s = b[0];
    const uint4 *yp = reinterpret_cast<const uint4 *>(y + p * 32);
    for (int q = 0; q < 4; ++q) {
        const uint4 v = yp[q];
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
        for (int k = 0; k < 4; ++k) {
            const float2 f = __bfloat1622float2(h[k]);
            s += f.x * w[8 * q + 2 * k] + f.y * w[8 * q + 2 * k + 1];
        }
    }
    r[p] = s;
}

// Mean squared error over the finite targets (count of them: ncount) and its
// backward through the head: dz[p, c] = dr w[c] (y > 0), dw[c] += dr y[p, c],
// db += dr, loss += (r - t)^2 / ncount.
__global__ void head_loss_backward_kernel(const bf16 *y, long long M, const float *w, const float *r,
                                          const float *target, float inv_count, bf16 *dz, float *dw, float *db,
                                          float *loss) {
    __shared__ float s_dw[32], s_db, s_loss;
    if (threadIdx.x < 32) s_dw[threadIdx.x] = 0.f;
    if (threadIdx.x == 0) s_db = s_loss = 0.f;
    __syncthreads();
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < M) {
        const float t = target[p];
        const float d = isnan(t) ? 0.f : r[p] - t;
        const float dr = 2.f * d * inv_count;
        atomicAdd(&s_loss, d * d * inv_count);
        atomicAdd(&s_db, dr);
        const uint4 *yp = reinterpret_cast<const uint4 *>(y + p * 32);
        uint4 *zp = reinterpret_cast<uint4 *>(dz + p * 32);
        for (int q = 0; q < 4; ++q) {
            const uint4 v = yp[q];
            const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
            uint4 o;
            __nv_bfloat162 *oh = reinterpret_cast<__nv_bfloat162 *>(&o);
            for (int k = 0; k < 4; ++k) {
                const float2 f = __bfloat1622float2(h[k]);
                const int c = 8 * q + 2 * k;
                atomicAdd(&s_dw[c], dr * f.x);
                atomicAdd(&s_dw[c + 1], dr * f.y);
                oh[k] = __floats2bfloat162_rn(f.x > 0.f ? dr * w[c] : 0.f, f.y > 0.f ? dr * w[c + 1] : 0.f);
            }
            zp[q] = o;
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) atomicAdd(dw + threadIdx.x, s_dw[threadIdx.x]);
    if (threadIdx.x == 0) {
        atomicAdd(db, s_db);
        atomicAdd(loss, s_loss);
    }
}

// Adam on fp32 master weights; writes the bf16 copy (if any) and clears the gradient.
__global__ void adam_kernel(float *w, float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2, bf16 *wb) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    g[i] = 0.f;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
}

// Weights of the input gradient: wt[ci, tap' * cout + co] = w[co, (8 - tap') * cin + ci].
__global__ void weight_flip_kernel(const bf16 *w, int cin, int cout, int kpad_in, int kpad_out, bf16 *wt) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)cin * kpad_out) return;
    const int ci = (int)(idx / kpad_out), k = (int)(idx - (long long)ci * kpad_out);
    bf16 val = __float2bfloat16_rn(0.f);
    if (k < 9 * cout) {
        const int tap = k / cout, co = k - (k / cout) * cout;
        val = w[(long long)co * kpad_in + (8 - tap) * cin + ci];
    }
    wt[idx] = val;
}

// Release epochs of the tiles of Riemann2 problems from predicted arrival
// times at block resolution (one value per 4x4 block): per instance, tiles of
// 8x8 points (2x2 blocks), release = 1 + floor(epochs * tmin / tmax_instance)
// - lag, at least 1; tmin the tile's smallest prediction.  One CTA per instance.
__global__ void release_kernel(const float *pred, int Hb, int Wb, int tile_blocks, float epochs, int lag,
                               uint16_t *release) {
    const int b = blockIdx.x;
    const float *P = pred + (long long)b * Hb * Wb;
    __shared__ float s_max[32];
    float mx = 0.f;
    for (int i = threadIdx.x; i < Hb * Wb; i += blockDim.x) {
        const float v = P[i];
        if (isfinite(v)) mx = fmaxf(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < blockDim.x / 32 ? s_max[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0) s_max[0] = v;
    }
    __syncthreads();
    const float tmax = s_max[0];
    const int To = Hb / tile_blocks, Tw = Wb / tile_blocks;
    for (int t = threadIdx.x; t < To * Tw; t += blockDim.x) {
        const int ty = t / Tw, tx = t - (t / Tw) * Tw;
        float mn = 3.4e38f;
        for (int dy = 0; dy < tile_blocks; ++dy)
            for (int dx = 0; dx < tile_blocks; ++dx) mn = fminf(mn, P[(ty * tile_blocks + dy) * Wb + tx * tile_blocks + dx]);
        float e = 1.f;
        if (tmax > 0.f && isfinite(mn)) e = 1.f + floorf(epochs * fmaxf(mn, 0.f) / tmax) - (float)lag;
        release[(long long)b * To * Tw + t] = (uint16_t)fminf(fmaxf(e, 1.f), 16000.f);
    }
}

// Warm-start values of Riemann2 problems in tile layout (8x8 tiles): (1 +
// margin) times the bilinear interpolation of the block predictions.
__global__ void warm_values_kernel(const float *pred, int n, int Hb, int Wb, int H, int W, float margin,
                                   float *values) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per = (long long)H * W;
    if (idx >= per * n) return;
    const int b = (int)(idx / per);
    const int r = (int)(idx - (long long)b * per);
    const int i = r / W, j = r - (r / W) * W;
    const float *P = pred + (long long)b * Hb * Wb;
    const float fy = fminf(fmaxf((i + 0.5f) / 4.f - 0.5f, 0.f), (float)(Hb - 1));
    const float fx = fminf(fmaxf((j + 0.5f) / 4.f - 0.5f, 0.f), (float)(Wb - 1));
    const int y0 = (int)fy, x0 = (int)fx;
    const int y1 = min(y0 + 1, Hb - 1), x1 = min(x0 + 1, Wb - 1);
    const float ay = fy - y0, ax = fx - x0;
    const float v = (1.f - ay) * ((1.f - ax) * P[y0 * Wb + x0] + ax * P[y0 * Wb + x1]) +
                    ay * ((1.f - ax) * P[y1 * Wb + x0] + ax * P[y1 * Wb + x1]);
    const int To = W / 8;
    const long long t = (long long)(i / 8) * To + j / 8;
    values[(long long)b * per + t * 64 + (i % 8) * 8 + (j % 8)] = (1.f + margin) * v;
}

}  // namespace unet
}  // namespace agd

// ------------------------------------------------------------------ C ABI --
using namespace agd;
using namespace agd::unet;

namespace {

cudaStream_t cs(agd_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

int num_sms() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

int launched(const char *what) {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AGD_STATUS_OK : set_cuda_error(what, e);
}

// Channels per CTA tile: at most 256, a multiple of 16, tiles of equal width.
int tile_n(int N, int *ntiles) {
    *ntiles = (N + 255) / 256;
    const int per = (N + *ntiles - 1) / *ntiles;
    return (per + 15) / 16 * 16;
}

bool check_srcs(const agd_conv *c, Src *s0, Src *s1) {
    if (!c || c->n <= 0 || c->H <= 0 || c->W <= 0 || !c->src[0].data) return false;
    for (int k = 0; k < 2; ++k) {
        const agd_conv_src &s = c->src[k];
        if (k == 1 && !s.data) continue;
        if (s.channels <= 0 || s.channels % 8 || (s.up != 0 && s.up != 1)) return false;
        if (s.up && (c->H % 2 || c->W % 2)) return false;
        if (reinterpret_cast<uintptr_t>(s.data) % 16) return false;
    }
    *s0 = {static_cast<const bf16 *>(c->src[0].data), c->src[0].channels, c->src[0].up};
    *s1 = c->src[1].data ? Src{static_cast<const bf16 *>(c->src[1].data), c->src[1].channels, c->src[1].up}
                         : Src{nullptr, 0, 0};
    return true;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); NULL if unavailable.
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// bf16 tiled map of `rank` dims (innermost first), swizzle by the inner box
// row (128 or 64 bytes).
bool make_map(CUtensorMap *map, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
              const cuuint32_t *box, int row_bytes) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, const_cast<void *>(base), dims, strides, box,
              es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The TMA-fed forward when the shapes allow it: 1 launched, 0 not applicable.
int conv_tma(const agd_conv *c, const void *w, const float *bias, int relu, void *out_bf16, float *out_f32,
             unsigned *err, cudaStream_t st, int *rc) {
    const agd_conv_src &s0 = c->src[0], &s1 = c->src[1];
    const bool two_in = s1.data != nullptr;
    if (s0.up || (two_in && s1.up) || s0.channels % 32 || (two_in && s1.channels % 32)) return 0;
    if (c->W > 128 || 128 % c->W || ((long long)c->H * c->W) % 128) return 0;
    TmaArgs g{};
    g.H = c->H;
    g.W = c->W;
    g.R = 128 / c->W;
    g.C0 = s0.channels;
    g.C1 = two_in ? s1.channels : 0;
    g.cb0 = g.C0 % 64 ? 32 : 64;
    g.cb1 = g.C1 % 64 ? 32 : 64;
    g.cin = g.C0 + g.C1;
    g.N = c->cout;
    g.BN = tile_n(g.N, &g.ntiles);
    g.kchunks = 9 * (g.C0 / g.cb0 + g.C1 / g.cb1);
    g.bias = bias;
    g.relu = relu;
    g.out_bf = static_cast<bf16 *>(out_bf16);
    g.out_f = out_f32;
    g.M = (long long)c->n * c->H * c->W;
    g.err = err;
    const long long mtiles = g.M / kBM;
    if (mtiles * g.ntiles > 0x7fffffffLL) return 0;
    g.mtiles = (int)mtiles;
    const int kpad = kpad_of(9 * g.cin);
    CUtensorMap xa0, xa1, wb64, wb32;
    const int ins = two_in ? 2 : 1;
    for (int k = 0; k < ins; ++k) {
        const agd_conv_src &sr = c->src[k];
        const int C = sr.channels, cb = C % 64 ? 32 : 64;
        const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)c->W, (cuuint64_t)c->H, (cuuint64_t)c->n};
        const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)c->W * C * 2, (cuuint64_t)c->H * c->W * C * 2};
        const cuuint32_t box[4] = {(cuuint32_t)cb, (cuuint32_t)c->W, (cuuint32_t)g.R, 1};
        if (!make_map(k ? &xa1 : &xa0, sr.data, 4, dims, strides, box, 2 * cb)) return 0;
    }
    if (!two_in) xa1 = xa0;
    const cuuint64_t wdims[2] = {(cuuint64_t)kpad, (cuuint64_t)g.N};
    const cuuint64_t wstr[1] = {(cuuint64_t)kpad * 2};
    const cuuint32_t box64[2] = {64, (cuuint32_t)g.BN}, box32[2] = {32, (cuuint32_t)g.BN};
    if (!make_map(&wb64, w, 2, wdims, wstr, box64, 128) || !make_map(&wb32, w, 2, wdims, wstr, box32, 64)) return 0;
    const bool two = g.BN <= 128;
    const int budget = (two ? kSmemBudget2 : kSmemBudget) - 1024;
    // small chunks (32-channel blocks, few output channels) share a stage, so
    // that a barrier round trip carries more tensor work
    g.rowmax = 2 * std::max(g.cb0, two_in ? g.cb1 : 0);
    g.spc = 1;
    const int slot = (kBM + g.BN) * g.rowmax;
    static const int spc_max = [] {
        const char *e = getenv("AGD_CONV_CHUNKS_PER_STAGE");  // tuning: 1, 2 or 4 (default 4)
        const int v = e ? atoi(e) : 4;
        return v == 1 || v == 2 ? v : 4;
    }();
    while (g.spc < spc_max && g.spc * 2 <= g.kchunks && (g.rowmax == 64 || g.BN <= 32) &&
           3 * slot * g.spc * 2 <= budget)
        g.spc *= 2;
    const int stage = slot * g.spc;
    g.stages = std::min(kMaxStages, budget / stage);
    if (g.stages < 2) return 0;
    const int smem = two ? g.stages * stage + 1024 : std::max(g.stages * stage + 1024, 120 * 1024);
    cudaError_t e = cudaFuncSetAttribute(conv_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) {
        *rc = set_cuda_error("conv3x3 shared memory", e);
        return 1;
    }
    const int grid = (int)std::min<long long>(mtiles * g.ntiles, (two ? 2 : 1) * num_sms());
    conv_tma_kernel<<<grid, kPThreads, smem, st>>>(g, xa0, xa1, wb64, wb32);
    *rc = launched("conv3x3 forward (TMA)");
    return 1;
}

}  // namespace

extern "C" {

int agd_conv_kpad(int cin) { return kpad_of(9 * cin); }

int agd_conv3x3_forward(const agd_conv *c, const void *w, const float *bias, int relu, void *out_bf16,
                        float *out_f32, unsigned *err, agd_stream_t stream) {
    GemmArgs g{};
    if (!check_srcs(c, &g.s0, &g.s1)) return set_error(AGD_STATUS_INVALID, "conv3x3: bad inputs");
    if (!w || !err || (!out_bf16) == (!out_f32) || c->cout <= 0 || c->cout % 16)
        return set_error(AGD_STATUS_INVALID, "conv3x3: weights, err, one output and cout % 16 == 0 are required");
    int rc = AGD_STATUS_OK;
    if (reinterpret_cast<uintptr_t>(w) % 16 == 0 && conv_tma(c, w, bias, relu, out_bf16, out_f32, err, cs(stream), &rc))
        return rc;
    g.nimg = c->n;
    g.H = c->H;
    g.W = c->W;
    const int cin = g.s0.C + g.s1.C;
    g.cin8 = cin / 8;
    g.K8 = 9 * g.cin8;
    g.kchunks = (g.K8 + 7) / 8;
    g.N = c->cout;
    GemmLaunch gl{};
    g.BN = tile_n(g.N, &gl.ntiles);
    g.wmat = static_cast<const bf16 *>(w);
    g.kpad = kpad_of(9 * cin);
    g.bias = bias;
    g.relu = relu;
    g.out_bf = static_cast<bf16 *>(out_bf16);
    g.out_f = out_f32;
    g.M = (long long)c->n * c->H * c->W;
    g.err = err;
    g.wshift = (c->W & (c->W - 1)) == 0 ? __builtin_ctz((unsigned)c->W) : -1;
    const long long mtiles = (g.M + kBM - 1) / kBM;
    if (mtiles * gl.ntiles > 0x7fffffffLL) return set_error(AGD_STATUS_INVALID, "conv3x3: too many pixels");
    gl.mtiles = (int)mtiles;
    const int a_bytes = kBM * kBK * 2, bchunk = g.BN * kBK * 2;
    const bool two = g.BN <= 128;  // two CTAs per SM: 2 x 2 x BN tensor memory columns
    const int budget = two ? kSmemBudget2 : kSmemBudget;
    gl.stationary = gl.ntiles == 1 && g.kchunks * bchunk <= budget / 2;
    const int stat = gl.stationary ? g.kchunks * bchunk : 0;
    const int stage = a_bytes + (gl.stationary ? 0 : bchunk);
    gl.stages = std::min(kMaxStages, (budget - stat) / stage);
    if (gl.stages < 2) return set_error(AGD_STATUS_UNSUPPORTED, "conv3x3: operands do not fit in shared memory");
    // a CTA alone on its SM asks for more than half of the shared memory
    const int smem = two ? gl.stages * stage + stat : std::max(gl.stages * stage + stat, 120 * 1024);
    cudaError_t e = cudaFuncSetAttribute(conv_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return set_cuda_error("conv3x3 shared memory", e);
    const int grid = (int)std::min<long long>(mtiles * gl.ntiles, (two ? 2 : 1) * num_sms());
    conv_gemm_kernel<<<grid, kPThreads, smem, cs(stream)>>>(g, gl);
    return launched("conv3x3 forward");
}

int agd_conv3x3_weight_grad(const agd_conv *c, const void *dz, float *dw, unsigned *err, agd_stream_t stream) {
    WgradArgs g{};
    if (!check_srcs(c, &g.s0, &g.s1)) return set_error(AGD_STATUS_INVALID, "conv3x3 weight grad: bad inputs");
    if (!dz || !dw || !err || c->cout <= 0 || c->cout % 16 || reinterpret_cast<uintptr_t>(dz) % 16)
        return set_error(AGD_STATUS_INVALID, "conv3x3 weight grad: dz, dw, err and cout % 16 == 0 are required");
    g.nimg = c->n;
    g.H = c->H;
    g.W = c->W;
    const int cin = g.s0.C + g.s1.C;
    g.cin8 = cin / 8;
    g.K8 = 9 * g.cin8;
    g.dz = static_cast<const bf16 *>(dz);
    g.N = c->cout;
    g.BN = tile_n(g.N, &g.ntiles);
    g.dw = dw;
    g.kpad = kpad_of(9 * cin);
    g.M = (long long)c->n * c->H * c->W;
    g.err = err;
    g.wshift = (c->W & (c->W - 1)) == 0 ? __builtin_ctz((unsigned)c->W) : -1;
    const long long nchunks = (g.M + kBK - 1) / kBK;
    if (nchunks > 0x7fffffffLL) return set_error(AGD_STATUS_INVALID, "conv3x3 weight grad: too many pixels");
    g.nchunks = (int)nchunks;
    g.mtiles = (g.K8 * 8 + kBM - 1) / kBM;
    const int nsm = num_sms();
    int splits = std::max(1, std::min(g.nchunks, (8 * nsm + g.mtiles * g.ntiles - 1) / (g.mtiles * g.ntiles)));
    g.chunks_per_split = (g.nchunks + splits - 1) / splits;
    g.splits = (g.nchunks + g.chunks_per_split - 1) / g.chunks_per_split;
    const int stage = kBM * kBK * 2 + g.BN * kBK * 2;
    const bool two = g.BN <= 128;
    g.stages = std::min(kMaxStages, (two ? kSmemBudget2 : kSmemBudget) / stage);
    const int smem = two ? g.stages * stage : std::max(g.stages * stage, 120 * 1024);
    cudaError_t e = cudaFuncSetAttribute(conv_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return set_cuda_error("conv3x3 weight grad shared memory", e);
    const int grid = std::min(g.mtiles * g.ntiles * g.splits, (two ? 2 : 1) * nsm);
    conv_wgrad_kernel<<<grid, kPThreads, smem, cs(stream)>>>(g);
    return launched("conv3x3 weight grad");
}

int agd_conv_weight_flip(int cin, int cout, const void *w, void *wt, agd_stream_t stream) {
    if (cin <= 0 || cout <= 0 || !w || !wt) return set_error(AGD_STATUS_INVALID, "weight flip: bad arguments");
    const long long n = (long long)cin * kpad_of(9 * cout);
    weight_flip_kernel<<<(unsigned)((n + 255) / 256), 256, 0, cs(stream)>>>(
        static_cast<const bf16 *>(w), cin, cout, kpad_of(9 * cin), kpad_of(9 * cout), static_cast<bf16 *>(wt));
    return launched("weight flip");
}

int agd_ws_features(const float *metric, const float *seeds, int nseeds, int n, int H, int W, float h, void *x0,
                    float *dref, agd_stream_t stream) {
    if (!metric || !seeds || nseeds <= 0 || n <= 0 || H % 8 || W % 8 || H <= 0 || W <= 0 || !x0 || !dref)
        return set_error(AGD_STATUS_INVALID, "features: bad arguments");
    const long long m = (long long)n * (H / 4) * (W / 4);
    features_kernel<<<(unsigned)((m + 255) / 256), 256, 0, cs(stream)>>>(metric, seeds, nseeds, n, H, W, h,
                                                                         static_cast<bf16 *>(x0), dref);
    return launched("features");
}

int agd_ws_target(const float *values, int n, int H, int W, const float *dref, float *target, agd_stream_t stream) {
    if (!values || !dref || !target || n <= 0 || H % 4 || W % 4) return set_error(AGD_STATUS_INVALID, "target: bad arguments");
    const long long m = (long long)n * (H / 4) * (W / 4);
    target_kernel<<<(unsigned)((m + 255) / 256), 256, 0, cs(stream)>>>(values, n, H, W, dref, target);
    return launched("target");
}

int agd_ws_avgpool(const void *x, int n, int H, int W, int C, void *y, agd_stream_t stream) {
    if (!x || !y || n <= 0 || H % 2 || W % 2 || C % 8) return set_error(AGD_STATUS_INVALID, "avgpool: bad arguments");
    const long long m = (long long)n * (H / 2) * (W / 2) * (C / 8);
    avgpool_kernel<<<(unsigned)((m + 255) / 256), 256, 0, cs(stream)>>>(static_cast<const bf16 *>(x), n, H, W, C,
                                                                        static_cast<bf16 *>(y));
    return launched("avgpool");
}

int agd_ws_upsample(const void *x, int n, int H, int W, int C, void *y, agd_stream_t stream) {
    if (!x || !y || n <= 0 || H <= 0 || W <= 0 || C % 8) return set_error(AGD_STATUS_INVALID, "upsample: bad arguments");
    const long long m = (long long)n * 4 * H * W * (C / 8);
    upsample_kernel<<<(unsigned)((m + 255) / 256), 256, 0, cs(stream)>>>(static_cast<const bf16 *>(x), n, H, W, C,
                                                                         static_cast<bf16 *>(y));
    return launched("upsample");
}

int agd_ws_route(int n, int H, int W, int C, const void *y, agd_ws_term t0, agd_ws_term t1, void *dz,
                 agd_stream_t stream) {
    if (!dz || n <= 0 || C <= 0) return set_error(AGD_STATUS_INVALID, "route: bad arguments");
    const agd_ws_term ts[2] = {t0, t1};
    for (const agd_ws_term &t : ts)
        if (t.mode < 0 || t.mode > 3 || (t.mode && (!t.data || t.offset + C > t.channels)))
            return set_error(AGD_STATUS_INVALID, "route: bad term");
    const long long m = (long long)n * H * W * C;
    route_kernel<<<(unsigned)((m + 255) / 256), 256, 0, cs(stream)>>>(
        n, H, W, C, static_cast<const bf16 *>(y), RouteTerm{t0.data, t0.mode, t0.channels, t0.offset},
        RouteTerm{t1.data, t1.mode, t1.channels, t1.offset}, static_cast<bf16 *>(dz));
    return launched("route");
}

int agd_ws_bias_grad(const void *dz, long long M, int C, float *db, agd_stream_t stream) {
    if (!dz || !db || M <= 0 || C <= 0 || C > 256) return set_error(AGD_STATUS_INVALID, "bias grad: bad arguments");
    const int threads = 256 / C * C;
    const long long blocks = std::min<long long>(1184, (M + 255) / 256);
    bias_grad_kernel<<<(unsigned)blocks, threads, 0, cs(stream)>>>(static_cast<const bf16 *>(dz), M, C, db);
    return launched("bias grad");
}

int agd_ws_head_forward(const void *y, long long M, const float *w, const float *b, float *r, agd_stream_t stream) {
    if (!y || !w || !b || !r || M <= 0) return set_error(AGD_STATUS_INVALID, "head: bad arguments");
    head_forward_kernel<<<(unsigned)((M + 255) / 256), 256, 0, cs(stream)>>>(static_cast<const bf16 *>(y), M, w, b, r);
    return launched("head forward");
}

int agd_ws_head_loss_backward(const void *y, long long M, const float *w, const float *r, const float *target,
                              long long ncount, void *dz, float *dw, float *db, float *loss, agd_stream_t stream) {
    if (!y || !w || !r || !target || !dz || !dw || !db || !loss || M <= 0 || ncount <= 0)
        return set_error(AGD_STATUS_INVALID, "head loss: bad arguments");
    head_loss_backward_kernel<<<(unsigned)((M + 255) / 256), 256, 0, cs(stream)>>>(
        static_cast<const bf16 *>(y), M, w, r, target, 1.f / (float)ncount, static_cast<bf16 *>(dz), dw, db, loss);
    return launched("head loss backward");
}

int agd_ws_adam(float *w, float *g, float *m, float *v, long long n, float lr, float beta1, float beta2, float eps,
                int t, void *wb, agd_stream_t stream) {
    if (!w || !g || !m || !v || n <= 0 || t < 1) return set_error(AGD_STATUS_INVALID, "adam: bad arguments");
    const float bc1 = 1.f - powf(beta1, (float)t), bc2 = 1.f - powf(beta2, (float)t);
    adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, cs(stream)>>>(w, g, m, v, n, lr, beta1, beta2, eps, bc1, bc2,
                                                                     static_cast<bf16 *>(wb));
    return launched("adam");
}

int agd_ws_release(const float *pred, int n, int Hb, int Wb, float epochs, int lag, uint16_t *release,
                   agd_stream_t stream) {
    if (!pred || !release || n <= 0 || Hb % 2 || Wb % 2 || !(epochs > 0.f))
        return set_error(AGD_STATUS_INVALID, "release: bad arguments");
    release_kernel<<<n, 256, 0, cs(stream)>>>(pred, Hb, Wb, 2, epochs, lag, release);
    return launched("release");
}

int agd_ws_warm_values(const float *pred, int n, int H, int W, float margin, float *values, agd_stream_t stream) {
    if (!pred || !values || n <= 0 || H % 8 || W % 8) return set_error(AGD_STATUS_INVALID, "warm values: bad arguments");
    const long long m = (long long)n * H * W;
    warm_values_kernel<<<(unsigned)((m + 255) / 256), 256, 0, cs(stream)>>>(pred, n, H / 4, W / 4, H, W, margin, values);
    return launched("warm values");
}

}  // extern "C"
