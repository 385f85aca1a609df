/*
 * agd_warmstart.h - C ABI of the learned warm start of the B200 eikonal path.
 *
 * The reference has no learned component: nothing here replaces reference
 * code.  A small U-Net (4 levels, 32 base channels, bf16 weights and
 * activations, fp32 accumulation) maps features of a Riemann2 problem (its
 * metric and seeds, at one value per 4x4 block of the grid) to the log-ratio
 * r = log(T / dref) of its block-mean arrival time T to the distance scale
 * dref; the solver uses the prediction through per-tile release epochs
 * (agd_instance.release) and warm-start values.
 *
 * Activations are NHWC bf16 (images, rows, columns, channels), channels a
 * multiple of 8.  Weights of a 3x3 convolution are a (cout, kpad) bf16 matrix,
 * column k = tap * cin + ci with tap = 3 (dy + 1) + (dx + 1), zero padded to
 * kpad = agd_conv_kpad(cin) columns.  All arrays are device memory owned by the
 * caller; nothing allocates.  Every call enqueues on `stream` and returns an
 * agd_status (agd_b200.h); `err` is a device word that a kernel sets when one
 * of its bounded waits gives up (0 on success, to be read by the caller).
 */
#ifndef AGD_WARMSTART_H
#define AGD_WARMSTART_H

#include <stddef.h>
#include <stdint.h>

#include "agd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* One input of a convolution: `channels` channels of an NHWC bf16 tensor at the
 * convolution's resolution (up = 0) or at half of it, read nearest-upsampled
 * (up = 1).  A convolution reads src[0]'s channels then src[1]'s (a
 * concatenation; src[1].data NULL when there is one input). */
typedef struct agd_conv_src {
    const void *data;
    int channels;
    int up;
} agd_conv_src;

typedef struct agd_conv {
    int n, H, W;            /* images, output (= input) rows and columns */
    agd_conv_src src[2];
    int cout;               /* output channels: a multiple of 16 */
} agd_conv;

/* Columns of a weight matrix with `cin` input channels: 9 cin rounded up to 64. */
int agd_conv_kpad(int cin);

/* out = act(conv3x3(inputs, w) + bias): an implicit GEMM on the tensor cores
 * (tcgen05.mma, fp32 accumulators in tensor memory), 128 pixels x up to 256
 * output channels per tile.  Inputs at the output's resolution with channel
 * counts that are multiples of 32, W dividing 128 and 128 dividing H W, are
 * moved by bulk tensor copies (TMA, swizzled tiles); other shapes by per-lane
 * cp.async gathers.  bias may be NULL; relu != 0 applies max(0, .).
 * Exactly one of out_bf16 (NHWC bf16) and out_f32 (NHWC fp32) is non NULL.
 * The input gradient of a convolution is this call on the output gradient with
 * the flipped weights of agd_conv_weight_flip, no bias, no ReLU, fp32 output. */
int agd_conv3x3_forward(const agd_conv *c, const void *w, const float *bias, int relu, void *out_bf16,
                        float *out_f32, unsigned *err, agd_stream_t stream);

/* dw += the weight gradient of the convolution c for the output gradient dz
 * ((n, H, W, cout) bf16): dw[co, tap cin + ci] += sum_p dz[p, co] x[p + tap, ci],
 * a GEMM over the pixels split across CTAs (tcgen05.mma with both operands
 * MN-major, as NHWC stores them); dw is fp32 (cout, kpad). */
int agd_conv3x3_weight_grad(const agd_conv *c, const void *dz, float *dw, unsigned *err, agd_stream_t stream);

/* Weights of the input gradient: wt (cin, agd_conv_kpad(cout)) bf16 with
 * wt[ci, tap' cout + co] = w[co, (8 - tap') cin + ci]. */
int agd_conv_weight_flip(int cin, int cout, const void *w, void *wt, agd_stream_t stream);

/* Features of n Riemann2 problems on an H x W grid (H, W multiples of 8, grid
 * scale h, origin 0): metric (n, H, W, 3) fp32 [m00, m10, m11], seeds (n,
 * nseeds, 2) domain coordinates.  x0: (n, H/4, W/4, 8) bf16; dref: (n, H/4,
 * W/4) fp32, the distance to the nearest seed plus 2h. */
int agd_ws_features(const float *metric, const float *seeds, int nseeds, int n, int H, int W, float h, void *x0,
                    float *dref, agd_stream_t stream);

/* Training target from solved values (n, H, W) fp32 grid layout:
 * log(block mean / dref), NaN where the mean is not finite. */
int agd_ws_target(const float *values, int n, int H, int W, const float *dref, float *target, agd_stream_t stream);

/* 2x2 average pooling, NHWC bf16 (n, H, W, C) -> (n, H/2, W/2, C). */
int agd_ws_avgpool(const void *x, int n, int H, int W, int C, void *y, agd_stream_t stream);

/* Nearest 2x upsampling, NHWC bf16 (n, H, W, C) -> (n, 2H, 2W, C): the decoder's
 * upsampled input materialised, so that its convolution can take the
 * bulk-copy operand path. */
int agd_ws_upsample(const void *x, int n, int H, int W, int C, void *y, agd_stream_t stream);

/* Gradient routing into a layer output y (n, H, W, C): the sum of up to two
 * fp32 NHWC terms (buffer, mode, buffer channels, channel offset): mode 1 the
 * same resolution, 2 the input gradient of a 2x2 average pool of y (buffer at
 * half resolution), 3 the input gradient of a nearest 2x upsampling of y
 * (buffer at double resolution); times the ReLU mask y > 0 (y NULL: none);
 * dz bf16 (n, H, W, C). */
typedef struct agd_ws_term {
    const float *data;
    int mode;
    int channels;
    int offset;
} agd_ws_term;
int agd_ws_route(int n, int H, int W, int C, const void *y, agd_ws_term t0, agd_ws_term t1, void *dz,
                 agd_stream_t stream);

/* db[c] += sum over the M pixels of dz[p, c] (dz bf16 (M, C), C <= 256). */
int agd_ws_bias_grad(const void *dz, long long M, int C, float *db, agd_stream_t stream);

/* 1x1 head over 32 channels: r[p] = sum_c y[p, c] w[c] + b[0]. */
int agd_ws_head_forward(const void *y, long long M, const float *w, const float *b, float *r, agd_stream_t stream);

/* Mean squared error of r against the finite entries of target (ncount of
 * them), added to *loss, and its backward through the head: dz = dr w (y > 0)
 * (bf16), dw += dr y, db += dr. */
int agd_ws_head_loss_backward(const void *y, long long M, const float *w, const float *r, const float *target,
                              long long ncount, void *dz, float *dw, float *db, float *loss, agd_stream_t stream);

/* Adam step on fp32 weights w with gradient g (cleared afterwards), moments m,
 * v; step t >= 1; wb (bf16 copy of w) may be NULL. */
int agd_ws_adam(float *w, float *g, float *m, float *v, long long n, float lr, float beta1, float beta2, float eps,
                int t, void *wb, agd_stream_t stream);

/* Release epochs of 8x8 tiles from block predictions of the arrival time
 * (n, Hb, Wb) fp32 (one value per 4x4 block): release = max(1, 1 +
 * floor(epochs tmin / tmax) - lag), tmin the tile's smallest prediction, tmax
 * the instance's largest.  release: (n, Hb/2, Wb/2) uint16, tile order. */
int agd_ws_release(const float *pred, int n, int Hb, int Wb, float epochs, int lag, uint16_t *release,
                   agd_stream_t stream);

/* Warm-start values of n H x W problems in 8x8 tile layout: (1 + margin) times
 * the bilinear interpolation of the block predictions (n, H/4, W/4). */
int agd_ws_warm_values(const float *pred, int n, int H, int W, float margin, float *values, agd_stream_t stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* AGD_WARMSTART_H */
