/* dsmc_surrogate.h - kernels of the field surrogate: a BF16 convolutional
 * encoder-decoder that maps a case (geometry mask and flow parameters on a
 * 128 x 128 canvas of the domain) to its sampled field (n, ux, uy, T).
 * The reference has no counterpart: it is the predictor of the warm start
 * (dsmc_init_warm).
 *
 * Tensors are NHWC with channel counts that are multiples of 32; activations
 * and weights are bfloat16 (passed as uint16_t bit patterns), accumulation
 * and optimizer state FP32.  Convolutions are 3 x 3, stride 1, zero padding
 * 1; weights are [Cout][3][3][Cin]; forward and input gradient, and the
 * weight gradient for Cin 32, 64 or 128 and Cout <= 256, run on the tcgen05
 * tensor cores (accumulator in tensor memory).  Every function enqueues on `stream`
 * (a cudaStream_t, NULL for the default stream) and returns DSMC_OK (0),
 * DSMC_ERR_ARGUMENT (2) for shapes outside these rules, or DSMC_ERR_CUDA (50).
 */
#ifndef DSMC_SURROGATE_H
#define DSMC_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y = act(conv(x, w) + bias) [+ res]: act is ReLU when relu != 0; res (same
 * shape as y, may be NULL) is added after the activation.  y (bf16) and/or
 * y32 (fp32) may be NULL.  Cin % 32 == 0, Cout % 32 == 0. */
int dsmc_sg_conv_fwd(const uint16_t *x, const uint16_t *w, const float *bias,
                     const uint16_t *res, uint16_t *y, float *y32, int n, int h, int w_,
                     int cin, int cout, int relu, void *stream);

/* A convolution with a skip connection: y = act(conv(x, w) + bias) and
 * ysum = y + skip, both bf16 (ysum from y as stored), in one pass. */
int dsmc_sg_conv_fwd_skip(const uint16_t *x, const uint16_t *w, const float *bias,
                          const uint16_t *skip, uint16_t *y, uint16_t *ysum, int n, int h,
                          int w_, int cin, int cout, int relu, void *stream);

/* dx = conv_transpose(dy, w): the input gradient of dsmc_sg_conv_fwd.
 * w_rot is scratch for the rotated weights, 9 * cin * cout elements. */
int dsmc_sg_conv_dgrad(const uint16_t *dy, const uint16_t *w, uint16_t *w_rot, uint16_t *dx,
                       int n, int h, int w_, int cin, int cout, void *stream);

/* The rotated weights dsmc_sg_conv_dgrad makes (w_rot[ci][8 - tap][co] =
 * w[co][tap][ci]) for `layers` (at most 32) layers in one launch: layer l
 * occupies elements offsets[l] (a multiple of 8) .. + 9 cin[l] cout[l] of
 * both w and w_rot.  dsmc_sg_conv_fwd(dy, w_rot + offsets[l], ..., cout[l],
 * cin[l], relu 0) is then that layer's input gradient. */
int dsmc_sg_rotate_layers(const uint16_t *w, uint16_t *w_rot, const int64_t *offsets,
                          const int *cin, const int *cout, int layers, void *stream);

/* dw += sum over pixels of dy (x) shifted x, FP32 [Cout][3][3][Cin];
 * db += sum over pixels of dy (db may be NULL; cout <= 256 with db).
 * Accumulates: clear first. */
int dsmc_sg_conv_wgrad(const uint16_t *dy, const uint16_t *x, float *dw, float *db, int n,
                       int h, int w_, int cin, int cout, void *stream);

/* dy *= (y > 0): the gradient through a ReLU whose output is y. */
int dsmc_sg_relu_bwd(uint16_t *dy, const uint16_t *y, int64_t count, void *stream);

/* One pass over a layer's output gradient dy (pixels x c, c a multiple of 8
 * up to 256): skip, when not NULL, receives dy as it comes (a copy, or
 * added when skip_accumulate); then dy *= (y > 0) when y is not NULL; then
 * db[ch] += the sum over pixels of dy[.][ch].  The relu, skip-gradient and
 * bias-gradient passes of a layer's backward step in one. */
int dsmc_sg_relu_bias_bwd(uint16_t *dy, const uint16_t *y, uint16_t *skip, int skip_accumulate,
                          float *db, int64_t pixels, int c, void *stream);

/* 2 x 2 average pooling (h, w even) and its gradient. */
int dsmc_sg_pool_fwd(const uint16_t *x, uint16_t *y, int n, int h, int w_, int c, void *stream);
int dsmc_sg_pool_bwd(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c,
                     void *stream);
/* The gradient added to dx (rounded to bf16 first) when accumulate. */
int dsmc_sg_pool_bwd_acc(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c,
                         int accumulate, void *stream);

/* Nearest 2x upsampling of an (n, h, w, c) tensor and its gradient. */
int dsmc_sg_up_fwd(const uint16_t *x, uint16_t *y, int n, int h, int w_, int c, void *stream);
int dsmc_sg_up_bwd(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c,
                   void *stream);
int dsmc_sg_up_bwd_acc(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c,
                       int accumulate, void *stream);

/* a += b elementwise (bf16). */
int dsmc_sg_add(uint16_t *a, const uint16_t *b, int64_t count, void *stream);

/* Masked mean squared error of the first `k` channels of out (fp32, c
 * channels, a multiple of 8) against target (fp32, k channels), weighted by mask (n*h*w,
 * 0 or 1); dy (bf16, c channels) receives its gradient (zero beyond k) and
 * loss[0] (device fp32) the loss.  Scaled by 1 / (k * sum of mask). */
int dsmc_sg_mse(const float *out, const float *target, const float *mask, uint16_t *dy,
                float *loss, int64_t pixels, int c, int k, void *stream);

/* One Adam step (Kingma and Ba, 2015, Algorithm 1) on FP32 master weights
 * with bias correction for step t (1-based); the bf16 copy is refreshed. */
int dsmc_sg_adam(float *w, uint16_t *w_bf16, const float *g, float *m, float *v, int64_t count,
                 float lr, float beta1, float beta2, float eps, int t, void *stream);

/* The same step with the learning rate and the bias corrections read from
 * device memory when the kernel runs: step = {lr, 1 - beta1^t, 1 - beta2^t}
 * (FP32), so that a step captured in a CUDA graph can be replayed with the
 * values of each step. */
int dsmc_sg_adam_dev(float *w, uint16_t *w_bf16, const float *g, float *m, float *v,
                     int64_t count, const float *step, float beta1, float beta2, float eps,
                     void *stream);

/* FP32 -> bf16 (round to nearest even). */
int dsmc_sg_to_bf16(const float *x, uint16_t *y, int64_t count, void *stream);

/* Synchronizes `stream`; returns 60 (a timeout) when a tensor-core kernel
 * gave up one of its bounded waits since the last check (and forgets it),
 * 50 on a CUDA error, else 0. */
int dsmc_sg_check(void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DSMC_SURROGATE_H */
