/*
 * cd_ops.h -- C ABI of the B200 (sm_100a) per-frame hot path of the online
 * cross-regression denoiser.
 *
 * Every entry point is stateless and stream ordered: it validates its
 * arguments on the host, enqueues kernels on `stream` and returns.  Nothing is
 * allocated behind the caller's back; ops that need scratch memory take a
 * caller-owned workspace whose size the matching *_workspace_size() call
 * reports.  Errors are returned as cd_status codes (never exit(), never
 * abort()); cd_get_last_error() returns a human-readable message for the most
 * recent failure on the calling host thread.
 *
 * Layout: every image is NHWC float32, contiguous, in device memory.  C = 3 for
 * colour, albedo, normal, motion vectors, linear depth and pn_fwidth; C = 5 for
 * band; C = 1 for opacity, variances, weight sums and success masks.  Boolean
 * masks are one byte per pixel (0 or 1), like TensorFlow's DT_BOOL.
 *
 * Each declaration cites the reference interface it replaces
 * (file:line inside the CGLab-GIST/cross-denoiser source tree).
 */
#ifndef CD_OPS_H
#define CD_OPS_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#if defined(__GNUC__)
#define CD_API __attribute__((visibility("default")))
#else
#define CD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cd_status {
    CD_OK = 0,
    /* An argument is out of range.  Covers the reference's OP_REQUIRES
       InvalidArgument checks (ops/regression.cc:134-135, 159-160) and the
       shapes on which the reference kernels would read or write out of bounds. */
    CD_EINVAL = 1,
    /* A CUDA runtime call or kernel launch failed (the reference calls exit(1)
       through CUDA_CHECK, ops/reproject.cc:23-30). */
    CD_ECUDA = 2,
    /* The caller's workspace is smaller than the *_workspace_size() figure. */
    CD_ENOMEM = 3
} cd_status;

/* Version of this ABI; bumped on any signature change. */
CD_API int cd_abi_version(void);

/* Message of the last failing call on this host thread ("" if none). */
CD_API const char *cd_get_last_error(void);

/* ------------------------------------------------------------------------ */
/* CrossRegression                                                           */
/* Replaces REGISTER_OP("CrossRegression") + CrossRegressionOp::Compute       */
/* (ops/regression.cc:25-57, 147-191) and CrossRegressionFunc                 */
/* (ops/regression.cu.cc:477-500).                                            */
/*                                                                            */
/*  imga, imgb, albedo, normal : [B,H,W,3]                                    */
/*  outa, outb                 : [B,H/recon_scale,W/recon_scale,3]            */
/*  vara, varb                 : [B,H,W,1]                                    */
/* outa is imgb regressed on imga's features, outb the converse; vara/varb    */
/* are the 3x3 leave-centre-out variance estimates of imga/imgb.              */
/* Requirements (CD_EINVAL otherwise): win_size >= 1, sparsity >= 1,          */
/* 1 <= recon_scale <= sparsity, H and W divisible by sparsity and by         */
/* recon_scale, win_size/2 < min(H, W).                                       */
/* The workspace holds the per-centre regression coefficients (the           */
/* reference's process-static betaA/betaB, ops/regression.cc:174-180) and    */
/* the per-pixel standard deviations of both images.                          */
/* ------------------------------------------------------------------------ */
CD_API size_t cd_cross_regression_workspace_size(int B, int H, int W, int sparsity);

CD_API cd_status cd_cross_regression(const float *imga, const float *imgb,
                              const float *albedo, const float *normal,
                              float *outa, float *outb, float *vara, float *varb,
                              int B, int H, int W,
                              int win_size, int sparsity, int recon_scale,
                              void *workspace, size_t workspace_bytes,
                              cudaStream_t stream);

/* CrossRegression with an FP64 fallback for ill-conditioned centres (no     */
/* counterpart in the reference).  Same as cd_cross_regression, except that  */
/* a centre/channel whose FP32 Cholesky pivots give a condition estimate     */
/* (max L_ii / min L_ii)^2 above cond_limit (> 0; 1e6 is the intended value) */
/* is factored and solved again in double from the same FP32 normal         */
/* equations, and *fallback_count (a device uint32, may be NULL) is          */
/* incremented once per such centre and channel.  Outputs differ from the   */
/* reference only at those centres.                                           */
CD_API cd_status cd_cross_regression_fp64_fallback(const float *imga, const float *imgb,
                              const float *albedo, const float *normal,
                              float *outa, float *outb, float *vara, float *varb,
                              int B, int H, int W,
                              int win_size, int sparsity, int recon_scale,
                              float cond_limit, unsigned int *fallback_count,
                              void *workspace, size_t workspace_bytes,
                              cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* CrossRegression backward (no counterpart in the reference, which          */
/* registers a gradient only for SpatialFilter, scripts/ops.py:23-32; the     */
/* reference's training step runs the regression outside its GradientTape,  */
/* scripts/main.py:259-261 vs 289).  The analytic derivative of               */
/* cd_cross_regression: given dL/d(outa, outb, vara, varb) it returns         */
/* dL/d(imga, imgb, albedo, normal).  grad_vara / grad_varb may be NULL       */
/* (no loss on the variances).  It recomputes the forward, so it needs only  */
/* the forward's inputs.  Same requirements as cd_cross_regression; the      */
/* workspace holds the recomputed coefficients, their Cholesky factors, the  */
/* reconstruction's outputs and weight sums, staged centre records and the   */
/* per-pixel partial gradients (with recon_scale 1: 378 floats per pixel at  */
/* sparsity 1, 76 at sparsity 4).                                             */
/*  grad_outa, grad_outb : [B,H/recon_scale,W/recon_scale,3]                  */
/*  grad_vara, grad_varb : [B,H,W,1] or NULL                                  */
/*  grad_imga, grad_imgb, grad_albedo, grad_normal : [B,H,W,3]                */
/* ------------------------------------------------------------------------ */
CD_API size_t cd_cross_regression_grad_workspace_size(int B, int H, int W, int sparsity,
                                                      int recon_scale);

CD_API cd_status cd_cross_regression_grad(const float *imga, const float *imgb,
                                          const float *albedo, const float *normal,
                                          const float *grad_outa, const float *grad_outb,
                                          const float *grad_vara, const float *grad_varb,
                                          float *grad_imga, float *grad_imgb,
                                          float *grad_albedo, float *grad_normal,
                                          int B, int H, int W,
                                          int win_size, int sparsity, int recon_scale,
                                          void *workspace, size_t workspace_bytes,
                                          cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Forward and backward of CrossRegression without the backward's recompute */
/* (no counterpart in the reference).  cd_cross_regression_keep computes    */
/* cd_cross_regression's four outputs (bit-identical) and leaves the        */
/* variances, standard deviations, coefficients, Cholesky factors and the   */
/* reconstruction's outputs and weight sums in a workspace of               */
/* cd_cross_regression_grad_workspace_size() bytes;                         */
/* cd_cross_regression_grad_kept then computes cd_cross_regression_grad's   */
/* result (bit-identical) from that workspace without recomputing the       */
/* forward.  Pass the same inputs, attributes and workspace to both, and    */
/* nothing else may write the workspace in between.                         */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_cross_regression_keep(const float *imga, const float *imgb,
                                          const float *albedo, const float *normal,
                                          float *outa, float *outb, float *vara, float *varb,
                                          int B, int H, int W,
                                          int win_size, int sparsity, int recon_scale,
                                          void *grad_workspace, size_t grad_workspace_bytes,
                                          cudaStream_t stream);

CD_API cd_status cd_cross_regression_grad_kept(const float *imga, const float *imgb,
                                               const float *albedo, const float *normal,
                                               const float *grad_outa, const float *grad_outb,
                                               const float *grad_vara, const float *grad_varb,
                                               float *grad_imga, float *grad_imgb,
                                               float *grad_albedo, float *grad_normal,
                                               int B, int H, int W,
                                               int win_size, int sparsity, int recon_scale,
                                               void *grad_workspace, size_t grad_workspace_bytes,
                                               cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* CrossRegression without a workspace (no counterpart in the reference).    */
/* For callers that cannot allocate device memory when the op runs: a       */
/* renderer's or engine's frame loop that owns all device memory through its */
/* own pool and forbids mid-frame allocations (cudaMalloc may synchronise the */
/* device or fail under memory pressure), or a plugin host that passes       */
/* tensors in but gives plugins no allocator.  Same arguments and results as */
/* cd_cross_regression, minus the workspace: the scratch lives in one        */
/* file-scope device array of CD_NOALLOC_SCRATCH_MIB MiB that the driver     */
/* allocates when the library is loaded on a device and keeps until the      */
/* process exits (enough for one 1920x1080 frame at sparsity 4).  Problems   */
/* needing more scratch than that (cd_cross_regression_workspace_size) fail  */
/* with CD_ENOMEM.  All calls share the array: calls whose kernels overlap   */
/* on the GPU race and must be serialised by the caller.  The first call on  */
/* a device looks up the array's device address and caches it; make it     */
/* before any stream capture.  The cache survives cudaDeviceReset, so do not */
/* call this entry point on a device after resetting it.  Invalid arguments  */
/* give CD_EINVAL as in cd_cross_regression, checked before the size.        */
/* Nothing in the array needs to start at zero.                              */
/* ------------------------------------------------------------------------ */
#define CD_NOALLOC_SCRATCH_MIB 40

CD_API size_t cd_cross_regression_noalloc_capacity(void);

CD_API cd_status cd_cross_regression_noalloc(const float *imga, const float *imgb,
                                              const float *albedo, const float *normal,
                                              float *outa, float *outb, float *vara, float *varb,
                                              int B, int H, int W,
                                              int win_size, int sparsity, int recon_scale,
                                              cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* SpatialFilter (forward)                                                    */
/* Replaces REGISTER_OP("SpatialFilter") + SpatialFilterOp::Compute           */
/* (ops/regression.cc:59-86, 242-281) and SpatialFilterFunc                   */
/* (ops/regression.cu.cc:502-517).                                            */
/*  imga, imgb, albedo, normal : [B,H,W,3];  band : [B,H,W,5]                 */
/*  out_acca, out_accb : [B,H,W,3];  out_wgtsuma, out_wgtsumb : [B,H,W,1]     */
/* Unlike the reference it stores no per-pixel band partials: the backward   */
/* below recomputes them.  Requirement: win_size/2 < min(H, W).              */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_spatial_filter(const float *imga, const float *imgb,
                            const float *albedo, const float *normal,
                            const float *band,
                            float *out_acca, float *out_accb,
                            float *out_wgtsuma, float *out_wgtsumb,
                            int B, int H, int W, int win_size,
                            cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* SpatialFilterGrad                                                          */
/* Replaces REGISTER_OP("SpatialFilterGrad") + SpatialFilterGradOp::Compute   */
/* (ops/regression.cc:88-103, 290-322), SpatialFilterGradFunc                 */
/* (ops/regression.cu.cc:519-534) and the Python gradient registration        */
/* (scripts/ops.py:23-32).  Same argument list as the reference op; the      */
/* images and band, which the reference passes but does not read, are used  */
/* here to recompute the filter weights.                                      */
/*  grad_acca, grad_accb : [B,H,W,3];  grad_wgtsuma, grad_wgtsumb : [B,H,W,1] */
/*  out_grad_band : [B,H,W,5]                                                 */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_spatial_filter_grad(const float *grad_acca, const float *grad_accb,
                                 const float *grad_wgtsuma, const float *grad_wgtsumb,
                                 const float *imga, const float *imgb,
                                 const float *albedo, const float *normal,
                                 const float *band, float *out_grad_band,
                                 int B, int H, int W, int win_size,
                                 cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* SpatialFilter with stored partials: the reference's design (its forward   */
/* keeps 2 x [B,H,W,16] floats of band partials for the gradient op,         */
/* ops/regression.cc:218-225), kept for the recompute-vs-store measurement.  */
/* partials: [B,H,W,32] floats (128 B/px) written by the forward and read by */
/* the gradient; results are those of cd_spatial_filter and                  */
/* cd_spatial_filter_grad bit for bit.                                        */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_spatial_filter_stored(const float *imga, const float *imgb,
                                          const float *albedo, const float *normal,
                                          const float *band,
                                          float *out_acca, float *out_accb,
                                          float *out_wgtsuma, float *out_wgtsumb,
                                          float *partials, int B, int H, int W, int win_size,
                                          cudaStream_t stream);
CD_API cd_status cd_spatial_filter_grad_stored(const float *grad_acca, const float *grad_accb,
                                               const float *grad_wgtsuma, const float *grad_wgtsumb,
                                               const float *partials, float *out_grad_band,
                                               int B, int H, int W, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Reproject                                                                  */
/* Replaces REGISTER_OP("Reproject") + ReprojectOp::Compute                   */
/* (ops/reproject.cc:34-69, 93-171) and ReprojectFunc                         */
/* (ops/reproject.cu.cc:240-273).                                             */
/*  mvec, linear_z, prev_linear_z, normal, prev_normal, pn_fwidth : [B,H,W,3] */
/*  opacity, prev_opacity : [B,H,W,1];  success : [B,H,W,1] bytes (0/1)       */
/*  input_list[i], output_list[i] : [B,H,W,channels[i]]                        */
/* input_list, output_list and channels are HOST arrays of n_list entries    */
/* (device pointers / channel counts); they travel in the kernel parameter   */
/* block, so no pointer table is copied to the device.                       */
/* Requirements: 1 <= n_list <= CD_REPROJECT_MAX_LIST, channels[i] >= 1.     */
/* ------------------------------------------------------------------------ */
#define CD_REPROJECT_MAX_LIST 8

CD_API cd_status cd_reproject(const float *mvec,
                       int n_list, const float *const *input_list,
                       const int *channels, float *const *output_list,
                       const float *linear_z, const float *prev_linear_z,
                       const float *normal, const float *prev_normal,
                       const float *pn_fwidth,
                       const float *opacity, const float *prev_opacity,
                       uint8_t *success,
                       int B, int H, int W, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* 3x3 erosion of the reprojection mask                                       */
/* Replaces tf.cast + tf.nn.erosion2d(SAME, all-ones 3x3) + 1 in             */
/* scripts/main.py:270-276: out = min over the in-bounds 3x3 window of        */
/* float(success).                                                            */
/*  success : [B,H,W,1] bytes;  out : [B,H,W,1] float                         */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_erode3x3(const uint8_t *success, float *out,
                      int B, int H, int W, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* TemporalScreening                                                          */
/* Replaces REGISTER_OP("TemporalScreening") + TemporalScreeningOp::Compute   */
/* (ops/temporal.cu.cc:204-287) and the TemporalScreening kernel (:57-198).  */
/*  current1, current2, prev, prev1, prev2 : [B,H,W,3]                        */
/*  reproj_success : [B,H,W,1] float                                          */
/*  output, output1, output2 : [B,H,W,3];  success : [B,H,W,1] float          */
/* Requirements: win_curr >= 1, win_prev >= 1.                                */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_temporal_screening(const float *current1, const float *current2,
                                const float *prev, const float *prev1,
                                const float *prev2, const float *reproj_success,
                                float *output, float *output1, float *output2,
                                float *success,
                                int B, int H, int W, int win_curr, int win_prev,
                                cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Erosion fused with temporal screening (one pass instead of           */
/* scripts/main.py:270-280's erosion2d followed by temporal_screening).       */
/* Results are identical to cd_erode3x3 followed by cd_temporal_screening;    */
/* the eroded mask is also written (eroded : [B,H,W,1] float) because the     */
/* aggregation step reads it (scripts/main.py:223).                           */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_erode_temporal_screening(const float *current1, const float *current2,
                                      const float *prev, const float *prev1,
                                      const float *prev2, const uint8_t *reproj_mask,
                                      float *eroded,
                                      float *output, float *output1, float *output2,
                                      float *success,
                                      int B, int H, int W, int win_curr, int win_prev,
                                      cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Input preparation: y1 = log1p(color), y2 = log1p(color2), the            */
/* prepare_input of scripts/main.py:207-212.  n = number of floats in each.  */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_prepare_input(const float *color, const float *color2, float *y1, float *y2,
                                  size_t n, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Aggregation loss, forward and backward                                     */
/* Replaces aggregation_loss (scripts/main.py:214-248) and the part of the    */
/* TensorFlow gradient (scripts/main.py:302) that flows into the spatial      */
/* filter's outputs and alpha.                                                */
/*  sum1, sum2, prev_out, label1, label2, prev_label1, prev_label2 : [B,H,W,3] */
/*  sumw1, sumw2, alpha, success, success_prev, opacity : [B,H,W,1]           */
/*  out_log (before expm1), out (max(0, expm1(out_log))), loss : [B,H,W,3]    */
/*  avg_loss : one float, mean of loss over B*H*W*3 elements                  */
/*  grad_sum1, grad_sum2 : [B,H,W,3]; grad_sumw1, grad_sumw2, grad_alpha      */
/*  : [B,H,W,1] -- dL/d(input) of L = avg_loss.  loss may be NULL.            */
/* The workspace holds per-CTA partial sums of the loss (the mean is reduced */
/* in a fixed order, so it is deterministic).                                 */
/* ------------------------------------------------------------------------ */
CD_API size_t cd_aggregation_workspace_size(int B, int H, int W);
CD_API cd_status cd_aggregation_loss(const float *sum1, const float *sumw1, const float *sum2,
                                     const float *sumw2, const float *alpha, const float *success,
                                     const float *success_prev, const float *prev_out,
                                     const float *opacity, const float *label1, const float *label2,
                                     const float *prev_label1, const float *prev_label2,
                                     float *out_log, float *out, float *loss, float *avg_loss,
                                     float *grad_sum1, float *grad_sumw1, float *grad_sum2,
                                     float *grad_sumw2, float *grad_alpha, int B, int H, int W,
                                     void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Spatial filter + aggregation loss + band gradient in one pass             */
/* The spatial_filter -> aggregation_loss -> SpatialFilterGrad sequence of    */
/* scripts/main.py:295-302 with the labels crossed as :283-286 sets them      */
/* (label1 = ols2, label2 = ols1, prev_label1 = prev_ols2, prev_label2 =      */
/* prev_ols1).  Same results as cd_spatial_filter, cd_aggregation_loss and    */
/* cd_spatial_filter_grad in sequence, without the filter sums leaving the   */
/* chip.  grad_band : [B,H,W,5] = dL/dband, grad_alpha : [B,H,W,1].          */
/* ------------------------------------------------------------------------ */
CD_API size_t cd_filter_aggregate_workspace_size(int B, int H, int W);
CD_API cd_status cd_filter_aggregate(const float *ols1, const float *ols2, const float *albedo,
                                     const float *normal, const float *band, const float *alpha,
                                     const float *success, const float *success_prev,
                                     const float *prev_out, const float *opacity,
                                     const float *prev_ols1, const float *prev_ols2,
                                     float *out_log, float *out, float *avg_loss, float *grad_band,
                                     float *grad_alpha, int B, int H, int W, int win_size,
                                     void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Kernel-predicting U-Net (replaces the Keras model of scripts/main.py:83-118 */
/* and its tf.GradientTape / optimizer.apply_gradients, :289-303).            */
/* Parameters: one flat fp32 buffer of cd_unet_param_count() = 31,414        */
/* floats, the model's trainable variables in order, each conv kernel in     */
/* Keras layout [kh][kw][cin][cout] (Conv2DTranspose: [1][1][cout][cin])     */
/* followed by its bias.  The convolutions run on the tensor cores with bf16 */
/* operands and fp32 accumulation; activations are kept in bf16 in the      */
/* workspace; the 1x1 head is fp32.  H and W must be multiples of 4.         */
/*  ols1, ols2, prev_out, albedo, normal : [B,H,W,3] (the concatenated input) */
/*  band : [B,H,W,5] = 1/(p^2 + 1e-4);  alpha : [B,H,W,1] = sigmoid(p)       */
/* cd_unet_backward needs the workspace of the cd_unet_forward of the same   */
/* frame and parameters; it writes dL/dparams (same layout) given dL/dband   */
/* and dL/dalpha.  The first int32 of the workspace is an error flag: 0     */
/* while every bounded wait of the tensor-core kernels completed; nonzero   */
/* after one ran out (1: a bulk copy into shared memory, 2: an MMA batch).  */
/* The caller zeroes the workspace once and tests the flag for != 0 (it is  */
/* never cleared by the library).  Once it is set, the outputs of that call */
/* and of every later call are invalid, and every later kernel of the       */
/* process is suspect: the timed-out CTA left while its copies or MMAs      */
/* could still be writing its shared memory or TMEM.                        */
/* ------------------------------------------------------------------------ */
CD_API size_t cd_unet_param_count(void);
CD_API size_t cd_unet_workspace_size(int B, int H, int W);

CD_API cd_status cd_unet_forward(const float *ols1, const float *ols2, const float *prev_out,
                                 const float *albedo, const float *normal, const float *params,
                                 float *band, float *alpha, int B, int H, int W,
                                 void *workspace, size_t workspace_bytes, cudaStream_t stream);

CD_API cd_status cd_unet_backward(const float *grad_band, const float *grad_alpha,
                                  const float *params, float *grad_params, int B, int H, int W,
                                  void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* Adam with Keras semantics (scripts/main.py:81, keras.optimizers.Adam):    */
/* m += (g - m)(1 - beta1); v += (g^2 - v)(1 - beta2);                       */
/* p -= lr sqrt(1 - beta2^t) / (1 - beta1^t) * m / (sqrt(v) + epsilon),     */
/* with t = *step + 1; *step is a device int32 (the optimizer's iteration    */
/* count, 0 before the first update) that the call then increments, so a    */
/* captured CUDA graph replays successive steps.                              */
CD_API cd_status cd_adam_update(float *params, const float *grads, float *m, float *v, int n,
                                int *step, float lr, float beta1, float beta2, float epsilon,
                                cudaStream_t stream);

/* One 3x3 'same' conv layer of the network through the same tensor-core    */
/* kernels (for layer-level checks).  x, y, dz: bf16 row-chunk planes         */
/* [B][H][C/8][W][8] (C rounded up to a multiple of 8; with C = 8 this is     */
/* NHWC), 16-byte aligned.  dgrad = 0: y = relu(conv(x) + bias),             */
/* x has cin channels, y cout; dgrad = 1: y = dL/dx given x = dL/dz (the     */
/* pre-activation gradient, cout channels), no bias, no ReLU.  cin in        */
/* {8, 15, 16, 24, 32, 48}, cout in {8, 16, 32}.                              */
CD_API size_t cd_unet_conv3x3_workspace_size(int cin, int cout);
CD_API cd_status cd_unet_conv3x3(const float *weight, const float *bias, const void *x, void *y,
                                 int cin, int cout, int dgrad, int B, int H, int W,
                                 void *workspace, size_t workspace_bytes, cudaStream_t stream);
/* Form of the 3x3 convolutions (forward and dgrad; no counterpart in the   */
/* reference), process-wide, read at the start of each call: 1 (default) =  */
/* ky-stacked for layers with 16 conv output channels (one MMA per input    */
/* row and K step accumulating into three output rows' accumulators; the   */
/* measured faster form there), one MMA per output row, tap and K step for  */
/* the others; 0 = one MMA per output row, tap and K step everywhere.       */
/* Same arithmetic per output (bf16 products, fp32 sums), sums in another   */
/* order.                                                                    */
CD_API void cd_set_unet_conv_stacked(int enable);
/* Weight and bias gradient of such a layer: grad = [dW (Keras layout), db]  */
/* from its input x (cin channels) and dz (cout channels).                    */
CD_API size_t cd_unet_conv3x3_wgrad_workspace_size(int cin, int cout, int B, int H, int W);
CD_API cd_status cd_unet_conv3x3_wgrad(const void *x, const void *dz, float *grad, int cin, int cout,
                                       int B, int H, int W, void *workspace, size_t workspace_bytes,
                                       cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* FP32 FMA throughput probe (no counterpart in the reference): `blocks`     */
/* CTAs of 256 threads each issue iters x 128 fused multiply-adds and store  */
/* one float per thread to out[blocks * 256].  Timed by the caller; gives    */
/* the measured FP32 peak that bounds the filter and regression kernels.     */
/* ------------------------------------------------------------------------ */
CD_API cd_status cd_fp32_fma_probe(float *out, int blocks, int iters, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Persistent kernels (no counterpart in the reference).  The fused erosion */
/* + temporal screening with win_prev = 1 runs as a persistent kernel that  */
/* stages its tiles by TMA and waits on an mbarrier with a bounded number   */
/* of polls, when the images' rows (and the mask's) are a multiple of 16    */
/* bytes and the tensors 16-byte aligned; the U-Net's convolutions with 16  */
/* outputs run as a persistent warp-specialised kernel (staging ring, MMA   */
/* thread, epilogue warps over two TMEM accumulator buffers) in the same    */
/* arithmetic order as the one-tile-per-CTA kernel.  Otherwise, or when     */
/* disabled here, the tile-per-CTA kernels run.  Both give the same results.*/
/* cd_image_kernel_error_flags: bit 0 = a screening staging wait ran out    */
/* (the tile's outputs are then not written); the bit only grows.  Read     */
/* synchronously; -1 if the read fails.                                     */
/* ------------------------------------------------------------------------ */
CD_API int cd_image_kernel_error_flags(void);
CD_API void cd_set_persistent_kernels(int enable);

/* ------------------------------------------------------------------------ */
/* Bounded-wait probe (no counterpart in the reference): one warp waits on  */
/* an mbarrier with the polling loop of the tensor-core kernels, for at     */
/* most max_iter polls (1 <= max_iter <= CD_MBAR_PROBE_MAX_ITER).  With      */
/* arrive = 0 nothing arrives, the wait runs out and *flag is set to 1;     */
/* with arrive = 1 the barrier completes and *flag is left unchanged.  No   */
/* copy or MMA is in flight, so the time-out leaves nothing behind.  Tests  */
/* the error path of cd_unet_forward/backward without a faulty kernel.      */
/* ------------------------------------------------------------------------ */
#define CD_MBAR_PROBE_MAX_ITER 65536
CD_API cd_status cd_mbar_timeout_probe(int *flag, int arrive, int max_iter, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* CD_OPS_H */
