// Internal interface of the U-Net kernels (unet_conv.cu, unet_ops.cu,
// unet.cu).  Activations are bf16 in row-chunk planes (below); parameters
// are fp32 masters in Keras layout, packed to bf16 tensor-core operands after
// every update.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cd {
namespace unet {

// Activation layout: [B][H][nch][W][8] bf16, nch = channels / 8 (channels
// padded to a multiple of 8 with zeros).  Each (row, chunk) is a contiguous
// plane of 16 bytes per pixel, so a row segment of one chunk is one bulk copy
// into the shared-memory chunk planes the tensor-core operands read, and a
// warp reading 32 consecutive pixels of a chunk reads 512 contiguous bytes.
// With nch = 1 this is NHWC.  Returns the index of pixel (b, y, x)'s chunk c
// in units of 8 channels.
__host__ __device__ inline size_t act_idx(int b, int y, int c, int x, int H, int W, int nch)
{
    return (((size_t)b * H + y) * nch + c) * W + x;
}

constexpr int kMaxSteps = 32;

// One K step of the implicit GEMM: staged input row offset ky, byte offset of
// the A view inside that row block (chunk plane + kx shift) and the byte
// distance to its second 16-channel half.
struct KStep {
    int ky, a_off, a_lbo, src;   // src: which input source's staged rows
};
// What each half of a K step multiplies: tap (ky, kx) of input chunk `chunk`
// (-1: unused, zero weights).  In a ky-stacked table (build_steps_stacked)
// ky is -1: the step's B operand holds the three vertical taps stacked along
// N (rows [0, n) ky = 2, [n, 2n) ky = 1, [2n, 3n) ky = 0).
struct StepHalf {
    int ky, kx, chunk;
};

struct ConvParams {
    const __nv_bfloat16 *src0, *src1;   // inputs, c0 and c1 chunks per pixel (concatenated)
    int c0, c1;
    const __nv_bfloat16 *wpack;         // packed B operand, nsteps * 2 * NOUT * 8 bf16
    const float *bias;                  // [NOUT] or null
    __nv_bfloat16 *dst0, *dst1;         // outputs, d0 and d1 chunks per pixel
    int d0, d1;
    const __nv_bfloat16 *mask0, *mask1; // ReLU masks laid out like dst0 / dst1, or null
    __nv_bfloat16 *pool;                // fused 2x2 max pool of dst0, or null
    int relu;
    int H, W, nsteps;
    int stacked;                        // 1: ky-stacked step table and B operand
    int *err;                           // set to 1 if an MMA wait times out
    KStep steps[kMaxSteps];
};

int build_steps(int c0, int c1, KStep *steps, StepHalf (*half)[2]);
// The same taps as build_steps with the three vertical taps of each (kx,
// chunk) pair in one step (a third of the steps, three times the B rows).
int build_steps_stacked(int c0, int c1, KStep *steps, StepHalf (*half)[2]);
// Process-wide choice of the convolution form (ky-stacked: one MMA per input
// row and K step feeds three output rows; per-row: one MMA per output row,
// tap and K step); set by cd_set_unet_conv_stacked, read once per call.
bool conv_stacked_enabled();
void set_conv_stacked(bool on);
cudaError_t launch_conv3x3(const ConvParams &P, int B, int nout, cudaStream_t st);

// Pack fp32 Keras weights W[3][3][cin][cout] into the B operand of a conv
// step table.  dgrad = 1 packs the flipped, transposed kernel (the conv of
// the output gradient): conv input channel = layer output channel.
struct PackTable {
    StepHalf half[kMaxSteps][2];
    int nsteps, nout, cin, cout, dgrad, stacked;   // stacked: 3 * nout B rows per half
};
cudaError_t launch_pack(const float *w, __nv_bfloat16 *dst, const PackTable &T, cudaStream_t st);

// Several layers' packing in one launch (one grid row per job).
constexpr int kMaxPackJobs = 12;
struct PackJob {
    const float *w;
    __nv_bfloat16 *dst;
    PackTable T;
};
struct PackJobs {
    PackJob job[kMaxPackJobs];
    int n;
};
cudaError_t launch_pack_jobs(const PackJobs &J, cudaStream_t st);

// Weight gradient of a 3x3 conv on the tensor cores: per CTA partial sums of
// dW[ky][kx][cin][cout] and db[cout] over its pixel tile.
struct WgradParams {
    const __nv_bfloat16 *x0, *x1;   // layer input (concatenated), xc0 + xc1 chunks
    int xc0, xc1;
    const __nv_bfloat16 *dz;        // pre-activation output gradient, zc chunks
    int zc;
    int cin, cout;                  // real channel counts
    float *partial;                 // [tiles][9 * cin * cout + cout]
    int H, W;
    int *err;
};
size_t wgrad_tiles(int B, int H, int W);
int wgrad_partial_rows(const WgradParams &P, int B);
size_t wgrad_partial_floats(int B, int H, int W, int cin, int cout);
cudaError_t launch_wgrad(const WgradParams &P, int B, cudaStream_t st);

// Whole network (unet.cu).  The first int32 of the workspace is an error flag
// that a kernel sets when a tensor-core wait times out.
int param_count();
size_t workspace_bytes(int B, int H, int W);
cudaError_t forward(const float *ols1, const float *ols2, const float *prev, const float *albedo,
                    const float *normal, const float *params, float *band, float *alpha, void *ws, int B, int H,
                    int W, cudaStream_t st);
cudaError_t backward(const float *gband, const float *galpha, const float *params, float *grads, void *ws, int B,
                     int H, int W, cudaStream_t st);
cudaError_t adam(float *w, const float *g, float *m, float *v, int n, int *step, float lr, float b1, float b2,
                 float eps, cudaStream_t st);

// Single 3x3 conv layer through the same kernels (layer tests): forward
// (bias + ReLU) or dgrad of a layer with cin -> cout channels.
cudaError_t conv_layer(const float *w, const float *bias, const __nv_bfloat16 *x, __nv_bfloat16 *y, int cin,
                       int cout, int dgrad, int B, int H, int W, void *ws, cudaStream_t st);
size_t conv_layer_workspace(int cin, int cout);
cudaError_t wgrad_layer(const __nv_bfloat16 *x, const __nv_bfloat16 *dz, float *grad, int cin, int cout, int B,
                        int H, int W, void *ws, cudaStream_t st);
size_t wgrad_layer_workspace(int cin, int cout, int B, int H, int W);

}  // namespace unet
}  // namespace cd
