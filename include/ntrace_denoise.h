/*
 * ntrace denoiser: a learned kernel-predicting filter for low-sample renders, C ABI.
 *
 * No counterpart in the reference (templeblock/math's painter only accumulates samples); the plain
 * render (nt_render) stays the fallback and the judge of the denoiser's error.  The network reads,
 * per pixel, the noisy mean radiance, the variance of that mean, the first-hit normal (n floats) and
 * depth, and a spatial noise estimate (from the mean's differences to the axis neighbours, defined
 * at one sample per pixel too), at the pixel and at its 2(n-1) neighbours along the screen axes,
 * and the input's noise level 1/sqrt(samples per pixel), and predicts for each
 * screen axis a cross-bilateral filter of 9 taps (-4..4): 9 tap logits and 3 log-bandwidths o_g of
 * the guides g (squared normal difference, squared depth difference, non-local-means colour distance
 * between the pixel and the tap); tap weight = softmax over taps of logit - sum_g
 * scale_g exp(min(o_g, 20)) D_g, scale = (4, 1, 0.05).  The filters are applied one axis after the
 * other to the noisy mean.  Layers: features -> 64 -> 64 -> 12(n-1), ReLU between, BF16 operands with
 * FP32 accumulation on the tensor cores (tcgen05), FP32 master weights trained with Adam on the loss
 * sum((out - target)^2) / sum((noisy - target)^2): the squared error left relative to the input's, so
 * that images of every noise level weigh alike in training.
 *
 * Inputs come from nt_render_moments and nt_render_aux (include/ntrace.h).  All image arrays are
 * device memory, pixels linear with x0 fastest, RGB as 3 floats per pixel.  Every function returns
 * an NT_* status (nt_last_error_message() for the text).  One denoiser must not be used by two
 * threads at once.
 */
#ifndef NTRACE_DENOISE_H
#define NTRACE_DENOISE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nt_denoiser nt_denoiser;

typedef struct nt_denoiser_layout
{
        int n;                /* space dimension (3..6); the screen has n-1 axes */
        int base_features;    /* per-pixel features: 3 mean + 3 std + n normal + 1 depth + 3 spatial noise = n + 10 */
        int features;         /* network inputs: base_features x (2(n-1) + 1), then the noise level */
        int features_padded;  /* inputs rounded up to a multiple of 16 (the MMA K step) */
        int hidden;           /* 64 */
        int outputs;          /* (9 + 3)(n-1): the 9 tap logits of every axis, then the 3 log-bandwidths of every axis */
        int outputs_padded;   /* rounded up to a multiple of 16 */
        int64_t param_count;  /* W1 (hidden x features), b1, W2 (hidden x hidden), b2, W3 (outputs x hidden), b3 */
} nt_denoiser_layout;

/* New network for n dimensions with seeded initial weights (Kaiming-uniform hidden layers, a small
 * output layer, zero biases). */
int nt_denoiser_create(int n, uint64_t seed, nt_denoiser** out);
int nt_denoiser_destroy(nt_denoiser* d);
int nt_denoiser_get_layout(nt_denoiser* d, nt_denoiser_layout* out);

/* FP32 master weights, param_count host floats in the order of nt_denoiser_layout. */
int nt_denoiser_get_params(nt_denoiser* d, float* params);
int nt_denoiser_set_params(nt_denoiser* d, const float* params);

/* The noisy image to work on: screen (n-1 ints), the samples per pixel it was rendered with (the
 * network reads 1/sqrt of it as the input's noise level), per-pixel mean (x3), variance of the mean
 * (x3), first-hit normal (x n) and depth (x1), all device arrays.  stream: a cudaStream_t or NULL (the
 * denoiser's own stream); every later call on this input uses the same stream. */
int nt_denoiser_set_input(nt_denoiser* d, const int32_t* screen, int samples_per_pixel, const float* d_mean,
                          const float* d_var, const float* d_normal, const float* d_depth, void* stream);

/* Denoised image of the current input into d_out (pixel_count x 3). */
int nt_denoiser_apply(nt_denoiser* d, float* d_out);

/* Loss against d_target (pixel_count x 3) and its gradient with respect to every parameter
 * (param_count host floats, may be NULL); the weights do not change. */
int nt_denoiser_gradient(nt_denoiser* d, const float* d_target, float* grad, double* loss);

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the loss against d_target; *loss (may be NULL)
 * is the loss before the step. */
int nt_denoiser_train_step(nt_denoiser* d, const float* d_target, float lr, double* loss);

/* The tensor-core GEMM the network runs on: C[M x N] = A[M x K] * B[N x K]^T with A and B row-major
 * BF16 (raw 16-bit patterns) and C row-major FP32, all device arrays; N and K multiples of 16,
 * N <= 256.  stream: a cudaStream_t or NULL (the default stream). */
int nt_tc_gemm_bf16(const uint16_t* d_a, const uint16_t* d_b, float* d_c, int m, int n, int k, void* stream);

/* The same GEMM in the form of the network's weight gradients: C[M x N] = At^T Bt with At (K x M) and
 * Bt (K x N) row-major BF16, i.e. both operands transposed (read MN-major), the K range split over CTAs
 * of k_per_cta each (0: one CTA per row block) whose partial sums are added into C with FP32 atomics
 * (C is zeroed first).  M a multiple of 8; N a multiple of 16, at most 256. */
int nt_tc_gemm_bf16_t(const uint16_t* d_at, const uint16_t* d_bt, float* d_c, int m, int n, int k, int k_per_cta,
                      void* stream);

/* Failure-detection self-test of the GEMM kernel: one small launch with its tensor-core instructions
 * withheld, so that the kernel's bounded wait for their completion (20 ms here, about a second in
 * ordinary launches) runs out; the kernel then gives its tensor memory back, raises its error flag and
 * returns.  Returns NT_ETIMEOUT when that happened as designed (the CUDA context stays usable), NT_OK if
 * the wait did not run out (a broken self-test), or another code on a CUDA error. */
int nt_tc_gemm_wait_selftest(void* stream);

#ifdef __cplusplus
}
#endif

#endif
