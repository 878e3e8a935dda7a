/* mdwt_denoiser.h -- C ABI of the learned denoiser of libmdwt.so.
 *
 * No counterpart in the reference renderer: the reference only accumulates frames
 * (deviceCode.cu:463-471).  The denoiser maps one low-spp frame's per-pixel features
 * (mdwt_set_features: radiance, depth, transmittance, channel hit fractions; 16 floats per
 * pixel) to a denoised RGB image, so that an image reaches a given RMSE with far fewer
 * path samples than plain accumulation; the plain accumulation stays the fallback, and
 * the error of both is measured the same way (mdwt_accum_rmse / mdwt_image_rmse).
 *
 * Network: a 3-level U-Net of 3x3 convolutions, 32/64/128 channels, ReLU, 2x2 average
 * pooling down, nearest 2x upsampling + skip concatenation up, a residual RGB output
 * (features.rgb + net).  BF16 weights and activations, FP32 accumulation, FP32 master
 * weights and Adam state; forward and backward on the GPU by the library's own kernels.
 * Sizes: any H x W (padded internally to multiples of 4).  Buffers passed as d_* are
 * device pointers on the denoiser's device; every call is asynchronous on `stream`
 * (NULL: the legacy default stream) except where a host result is returned.
 */
#ifndef MDWT_DENOISER_H
#define MDWT_DENOISER_H

#include <stdint.h>

#include "mdwt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mdwt_denoiser mdwt_denoiser;

/* He-initialised weights from `seed` (the output layer scaled by 0.1). */
mdwt_status mdwt_denoiser_create(mdwt_denoiser **out, int device, uint64_t seed);
mdwt_status mdwt_denoiser_destroy(mdwt_denoiser *d);
const char *mdwt_denoiser_last_error(const mdwt_denoiser *d);

/* Parameter vector: per layer (in network order) W[tap][co][ci] then bias[co], FP32. */
int64_t mdwt_denoiser_num_params(void);
mdwt_status mdwt_denoiser_get_params(mdwt_denoiser *d, float *host_out);
mdwt_status mdwt_denoiser_set_params(mdwt_denoiser *d, const float *host_in);

/* d_out_rgba [n][h][w][4] = denoised RGB, alpha 1, from d_features [n][h][w][16]. */
mdwt_status mdwt_denoiser_infer(mdwt_denoiser *d, const float *d_features, float *d_out_rgba, int n, int h, int w,
                                void *stream);
/* Loss = mean over n*h*w*3 of (denoised - target.rgb)^2, target [n][h][w][4]; gradients of
 * every parameter into the denoiser's gradient buffer (no update).  *loss (optional)
 * makes the call synchronous. */
mdwt_status mdwt_denoiser_backward(mdwt_denoiser *d, const float *d_features, const float *d_target_rgba, int n,
                                   int h, int w, double *loss, void *stream);
mdwt_status mdwt_denoiser_get_grads(mdwt_denoiser *d, float *host_out);
/* backward + one Adam step (beta 0.9 / 0.999, eps 1e-8) with learning rate lr. */
mdwt_status mdwt_denoiser_train_step(mdwt_denoiser *d, const float *d_features, const float *d_target_rgba, int n,
                                     int h, int w, float lr, double *loss, void *stream);
/* The pieces of a data-parallel training step (one process per GPU): backward on the
 * rank's shard, copy_grads into a vector of num_params floats (get_params order; device or
 * host memory), an all-reduce that averages it over the ranks, load_grads, adam_step.
 * copy_grads / load_grads are asynchronous on `stream`; adam_step is the update of
 * train_step, applied to the current gradient buffer. */
mdwt_status mdwt_denoiser_copy_grads(mdwt_denoiser *d, float *out, void *stream);
mdwt_status mdwt_denoiser_load_grads(mdwt_denoiser *d, const float *in, void *stream);
mdwt_status mdwt_denoiser_adam_step(mdwt_denoiser *d, float lr, void *stream);

/* Convolution path: 1 (default) = tcgen05 tensor-core kernels (persistent, warp-specialised;
 * two TMEM accumulators, so a tile's epilogue overlaps the next tile's MMAs) wherever the
 * layer shapes allow; 2 = the same kernels with one accumulator and the most rows per tile;
 * 0 = the mma.sync kernels everywhere.  The tiling is process-wide. */
mdwt_status mdwt_denoiser_set_tensor_cores(mdwt_denoiser *d, int mode);
/* Autotuner of the tensor-core convolutions for one input shape: every layer's candidate
 * tilings (output rows per CTA, input-channel chunk, weight stages) are timed on the real
 * operands of a forward pass on d_features [n][h][w][16] (and, with backward != 0, the
 * data gradients); the fastest are used for that shape until another is tuned.
 * Synchronous; results do not depend on the tiling beyond FP32 summation order. */
mdwt_status mdwt_denoiser_autotune(mdwt_denoiser *d, const float *d_features, int n, int h, int w, int backward);
/* Wait for the denoiser's work; MDWT_ERR_TIMEOUT when a tensor-core kernel's bounded
 * wait for its operands gave up (its output is then invalid).  The error is reported once
 * (the flag is cleared). */
mdwt_status mdwt_denoiser_check(mdwt_denoiser *d);
/* Test hook of the failure path (process-wide): the next `launches` tensor-core
 * convolutions issue no operand loads, so every CTA's bounded wait gives up after about a
 * second of SM clocks, the kernel exits cleanly and mdwt_denoiser_check reports
 * MDWT_ERR_TIMEOUT.  No GPU fault is involved.  0 cancels. */
mdwt_status mdwt_denoiser_test_stall(mdwt_denoiser *d, int launches);

/* Denoise the last frame of a render context (its features must be on) into
 * d_out_rgba [H][W][4] on the context's stream. */
mdwt_status mdwt_denoise(mdwt_ctx *ctx, mdwt_denoiser *d, float *d_out_rgba);
/* RMSE of an RGBA image [H][W][4] on the context's device against the context's FP64
 * expected image (mdwt_render_expected first); synchronous. */
mdwt_status mdwt_image_rmse(mdwt_ctx *ctx, const float *d_rgba, double *rmse);

#ifdef __cplusplus
}
#endif

#endif
