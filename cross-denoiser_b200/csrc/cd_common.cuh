// Shared device helpers for the sm_100a kernels of the per-frame hot path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define CD_DEV __device__ __forceinline__

namespace cd {

// Reflect-101 index of the regression and spatial-filter windows
// (ops/regression.cu.cc:128-129, 413-414).  Valid while the window radius is
// below the image extent, which the host side enforces.
CD_DEV int mirror(int i, int n) { return (i >= n) ? 2 * n - 2 - i : abs(i); }

// Ceil-division with C's truncating '/' and '%' (ops/cuda_utils.cuh:275-278);
// for negative a it is one above the mathematical ceiling when a % b != 0.
CD_DEV int idivup(int a, int b) { return (a % b != 0) ? (a / b + 1) : (a / b); }

CD_DEV float3 ld3(const float *p, size_t i)
{
    return make_float3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
}

CD_DEV void st3(float *p, size_t i, float3 v)
{
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

// x*x + y*y + z*z in the reference's source order (ops/cuda_utils.cuh:171-174).
CD_DEV float norm2(float x, float y, float z) { return x * x + y * y + z * z; }

}  // namespace cd

// Launchers implemented by the kernel translation units; each returns the
// result of cudaGetLastError() after its launches.
namespace cd {

cudaError_t launch_variance(const float *imga, const float *imgb, float *vara, float *varb,
                            float *sda, float *sdb, int B, int H, int W, cudaStream_t st);
cudaError_t launch_regression(const float *imga, const float *imgb, const float *albedo,
                              const float *normal, const float *vara, const float *varb,
                              const float *sda, const float *sdb, float *beta, int B, int H, int W,
                              int win, int sparsity, cudaStream_t st, float *chol = nullptr,
                              float cond_limit = 0.f, unsigned *fallbacks = nullptr);
cudaError_t launch_recon(const float *imga, const float *imgb, const float *albedo,
                         const float *normal, const float *vara, const float *varb,
                         const float *sda, const float *sdb, const float *beta, float *outa,
                         float *outb, int B, int H, int W, int win, int sparsity, int recon_scale,
                         cudaStream_t st, float *state = nullptr);
size_t regression_smem_bytes(int win, int sparsity);
// CrossRegression backward (regression_grad.cu); ws holds
// regression_grad_workspace_floats() floats.
size_t regression_grad_workspace_floats(int B, int H, int W, int sparsity, int recon_scale);
// kept: the workspace already holds the forward's quantities, written by
// launch_regression_keep (the forward's outputs plus those quantities).
cudaError_t launch_regression_grad(const float *imga, const float *imgb, const float *albedo,
                                   const float *normal, const float *g_outa, const float *g_outb,
                                   const float *g_vara, const float *g_varb, float *g_imga,
                                   float *g_imgb, float *g_albedo, float *g_normal, int B, int H,
                                   int W, int win, int sparsity, int recon_scale, float *ws,
                                   cudaStream_t st, bool kept = false);
cudaError_t launch_regression_keep(const float *imga, const float *imgb, const float *albedo,
                                   const float *normal, float *outa, float *outb, float *vara,
                                   float *varb, int B, int H, int W, int win, int sparsity,
                                   int recon_scale, float *ws, cudaStream_t st);
size_t recon_smem_bytes(int win, int sparsity, int recon_scale);

size_t spatial_filter_smem_bytes(int win);
cudaError_t launch_spatial_filter(const float *imga, const float *imgb, const float *albedo,
                                  const float *normal, const float *band, float *acca,
                                  float *accb, float *wsa, float *wsb, int B, int H, int W,
                                  int win, cudaStream_t st);
cudaError_t launch_spatial_filter_grad(const float *gacca, const float *gaccb, const float *gwsa,
                                       const float *gwsb, const float *imga, const float *imgb,
                                       const float *albedo, const float *normal,
                                       const float *band, float *gband, int B, int H, int W,
                                       int win, cudaStream_t st);

cudaError_t launch_spatial_filter_store(const float *imga, const float *imgb, const float *albedo,
                                        const float *normal, const float *band, float *acca, float *accb,
                                        float *wsa, float *wsb, float *partials, int B, int H, int W, int win,
                                        cudaStream_t st);
cudaError_t launch_spatial_filter_grad_stored(const float *gacca, const float *gaccb, const float *gwsa,
                                              const float *gwsb, const float *partials, float *gband, int B, int H,
                                              int W, cudaStream_t st);

struct ReprojectList {
    const float *in[8];
    float *out[8];
    int ch[8];
    int n;
};
cudaError_t launch_reproject(const float *mvec, const ReprojectList &list, const float *linz,
                             const float *plinz, const float *nrm, const float *pnrm,
                             const float *pnfw, const float *opac, const float *popac,
                             uint8_t *success, int B, int H, int W, cudaStream_t st);

cudaError_t launch_erode3x3(const uint8_t *mask, float *out, int B, int H, int W, cudaStream_t st);
cudaError_t launch_temporal(const float *c1, const float *c2, const float *prev,
                            const float *prev1, const float *prev2, const float *rs,
                            const uint8_t *raw_mask, float *eroded, float *out, float *out1,
                            float *out2, float *succ, int B, int H, int W, int win_curr,
                            int win_prev, cudaStream_t st);

// Sticky error bits of the persistent TMA image kernels (a staging wait ran
// out), read synchronously; -1 if the read fails.
int temporal_error_flag();

// Records msg as the calling thread's cd_get_last_error() message.
void set_last_error(const char *msg);
// The argument checks of cd_cross_regression (null pointers, shape and
// attributes); sets the last-error message and returns CD_EINVAL on failure.
int check_cross_regression_args(const char *op, const float *imga, const float *imgb, const float *albedo,
                                const float *normal, const float *outa, const float *outb, const float *vara,
                                const float *varb, int B, int H, int W, int win_size, int sparsity,
                                int recon_scale);

struct AggArgs {
    const float *s1, *w1, *s2, *w2, *alpha, *succ, *succ_prev, *prev, *opac, *l1, *l2, *pl1, *pl2;
    float *out_log, *out, *loss, *g_s1, *g_w1, *g_s2, *g_w2, *g_alpha;
};
size_t aggregation_partials(int B, int H, int W);
cudaError_t launch_log1p(const float *a, const float *b, float *ya, float *yb, size_t n, cudaStream_t st);
cudaError_t launch_aggregation(const AggArgs &A, float *partial, float *avg, int B, int H, int W,
                               cudaStream_t st);
size_t filter_aggregate_smem(int win);
cudaError_t launch_filter_aggregate(const float *imga, const float *imgb, const float *albedo,
                                    const float *normal, const float *band, const AggArgs &A,
                                    float *gband, float *partial, float *avg, int B, int H, int W,
                                    int win, cudaStream_t st);

}  // namespace cd
