// Launchers of the U-Net's non-convolution kernels (unet_ops.cu).  Activation
// tensors are bf16 row-chunk planes (unet.cuh).
#pragma once
#include <cstddef>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cd {
namespace unet {

cudaError_t launch_pack_input(const float *a, const float *b, const float *c, const float *d, const float *e,
                              __nv_bfloat16 *x, size_t n, int W, cudaStream_t st);
cudaError_t launch_tconv_fwd(int ci, int co, const __nv_bfloat16 *in, const float *K, const float *bias,
                             __nv_bfloat16 *out, int Hi, int Wi, int B, cudaStream_t st);
size_t tconv_blocks(int ci, int Hi, int Wi, int B);
cudaError_t launch_tconv_bwd(int ci, int co, const __nv_bfloat16 *in, const __nv_bfloat16 *dout, const float *K,
                             __nv_bfloat16 *dz_in, float *partial, int Hi, int Wi, int B, cudaStream_t st);
cudaError_t launch_head_fwd(const __nv_bfloat16 *x, const float *K, const float *bias, float *band, float *alpha,
                            size_t n, cudaStream_t st);
size_t head_blocks(size_t n);
cudaError_t launch_head_bwd(const __nv_bfloat16 *x, const float *K, const float *bias, const float *gband,
                            const float *galpha, __nv_bfloat16 *dz, float *partial, size_t n, cudaStream_t st);
cudaError_t launch_pool_bwd(int C, const __nv_bfloat16 *act, const __nv_bfloat16 *pooled,
                            const __nv_bfloat16 *dpool, const __nv_bfloat16 *dskip, __nv_bfloat16 *dz, int H, int W,
                            int B, cudaStream_t st);
// Sum per-tile partials partial[t * n + j] over t into out[j] (fixed order).
// The partial buffer holds reduce_floats(n, tiles) floats.
size_t reduce_floats(int n, int tiles);
cudaError_t launch_reduce(float *partial, float *out, int n, int tiles, cudaStream_t st);
cudaError_t launch_adam(float *w, const float *g, float *m, float *v, int n, int *step, float lr, float b1, float b2,
                        float eps, cudaStream_t st);

}  // namespace unet
}  // namespace cd
