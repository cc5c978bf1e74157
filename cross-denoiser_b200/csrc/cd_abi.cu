// C ABI of the per-frame hot path (declared in include/cd_ops.h).
//
// Every entry point validates its arguments on the host, enqueues its
// kernels on the caller's stream and reports failures as cd_status codes
// with a thread-local message; nothing here exits, allocates device memory or
// synchronises.  The argument checks mirror the reference op wrappers'
// OP_REQUIRES checks (ops/regression.cc:134-135, 159-160) and reject the
// shapes on which the reference kernels would index out of bounds.
#include <cstdarg>
#include <cstdio>
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "unet.cuh"
#include "tma.cuh"
#include "../../include/cd_ops.h"

namespace {

thread_local char g_err[512] = "";

cd_status fail(cd_status s, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return s;
}

cd_status cuda_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return CD_OK;
    return fail(CD_ECUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

bool dims_ok(int B, int H, int W) { return B >= 1 && B <= 32767 && H >= 1 && W >= 1 && H <= 65535 * 8 && W <= (1 << 24); }

// Shared-memory footprints of the tiled kernels (must agree with the kernel
// translation units; checked here so that an oversized window is an argument
// error rather than a launch failure).
size_t temporal_tile_bytes(int hc)
{
    return ((size_t)6 * (32 + 2 * hc) * (8 + 2 * hc) + (size_t)18 * (8 + 2 * hc) * 32) * 4;
}
constexpr size_t kSmemLimit = 220 * 1024;

}  // namespace

namespace cd {
void set_last_error(const char *msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }
}  // namespace cd

extern "C" {

int cd_abi_version(void) { return 1; }

int cd_image_kernel_error_flags(void)
{
    const int t = cd::temporal_error_flag();
    return t < 0 ? -1 : (t ? 1 : 0);
}

void cd_set_persistent_kernels(int enable) { cd::tma::set_persistent_enabled(enable != 0); }

void cd_set_unet_conv_stacked(int enable) { cd::unet::set_conv_stacked(enable != 0); }

const char *cd_get_last_error(void) { return g_err; }

size_t cd_cross_regression_workspace_size(int B, int H, int W, int sparsity)
{
    if (!dims_ok(B, H, W) || sparsity < 1) return 0;
    // coefficients of both buffers, then sqrt(var) of both images
    return ((size_t)2 * B * (H / sparsity) * (W / sparsity) * 18 + (size_t)2 * B * H * W) * sizeof(float);
}

// Shape and attribute checks shared by CrossRegression's forward and backward.
static cd_status check_regression(const char *op, int B, int H, int W, int win_size, int sparsity, int recon_scale)
{
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "%s: bad shape B=%d H=%d W=%d", op, B, H, W);
    if (win_size < 1 || sparsity < 1 || recon_scale < 1)
        return fail(CD_EINVAL, "%s: win_size, sparsity and recon_scale must be >= 1", op);
    if (recon_scale > sparsity)
        return fail(CD_EINVAL, "recon_scale must be less than or equal to sparsity");
    if (H % recon_scale != 0 || W % recon_scale != 0)
        return fail(CD_EINVAL, "Image height and width must be divisible by recon_scale");
    if (H % sparsity != 0 || W % sparsity != 0)
        return fail(CD_EINVAL, "%s: image height and width must be divisible by sparsity "
                               "(got %dx%d, sparsity %d)", op, H, W, sparsity);
    const int hw = win_size / 2;
    if (hw >= H || hw >= W)
        return fail(CD_EINVAL, "%s: window radius %d must be smaller than the image (%dx%d)", op, hw, H, W);
    if (cd::regression_smem_bytes(win_size, sparsity) > kSmemLimit ||
        cd::recon_smem_bytes(win_size, sparsity, recon_scale) > kSmemLimit)
        return fail(CD_EINVAL, "%s: win_size %d with sparsity %d / recon_scale %d exceeds the "
                               "shared-memory tiles", op, win_size, sparsity, recon_scale);
    return CD_OK;
}

}  // extern "C"

namespace cd {
int check_cross_regression_args(const char *op, const float *imga, const float *imgb, const float *albedo,
                                const float *normal, const float *outa, const float *outb, const float *vara,
                                const float *varb, int B, int H, int W, int win_size, int sparsity,
                                int recon_scale)
{
    if (!imga || !imgb || !albedo || !normal || !outa || !outb || !vara || !varb)
        return fail(CD_EINVAL, "%s: null tensor pointer", op);
    return check_regression(op, B, H, W, win_size, sparsity, recon_scale);
}
}  // namespace cd

extern "C" {

static cd_status cross_regression_impl(const char *op, const float *imga, const float *imgb, const float *albedo,
                                       const float *normal, float *outa, float *outb, float *vara, float *varb,
                                       int B, int H, int W, int win_size, int sparsity, int recon_scale,
                                       float cond_limit, unsigned *fallbacks, void *workspace,
                                       size_t workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    cd_status s = static_cast<cd_status>(cd::check_cross_regression_args(
        op, imga, imgb, albedo, normal, outa, outb, vara, varb, B, H, W, win_size, sparsity, recon_scale));
    if (s != CD_OK) return s;
    const size_t need = cd_cross_regression_workspace_size(B, H, W, sparsity);
    if (workspace_bytes < need || (need > 0 && !workspace))
        return fail(CD_ENOMEM, "%s: workspace of %zu bytes needed, %zu given", op, need, workspace_bytes);

    float *beta = static_cast<float *>(workspace);
    float *sda = beta + (size_t)2 * B * (H / sparsity) * (W / sparsity) * 18;
    float *sdb = sda + (size_t)B * H * W;
    if ((s = cuda_status(cd::launch_variance(imga, imgb, vara, varb, sda, sdb, B, H, W, stream), "variance")) != CD_OK)
        return s;
    if ((s = cuda_status(cd::launch_regression(imga, imgb, albedo, normal, vara, varb, sda, sdb, beta, B, H, W,
                                               win_size, sparsity, stream, nullptr, cond_limit, fallbacks),
                         "regression")) != CD_OK)
        return s;
    return cuda_status(cd::launch_recon(imga, imgb, albedo, normal, vara, varb, sda, sdb, beta, outa, outb, B,
                                        H, W, win_size, sparsity, recon_scale, stream), "recon");
}

cd_status cd_cross_regression(const float *imga, const float *imgb, const float *albedo,
                              const float *normal, float *outa, float *outb, float *vara,
                              float *varb, int B, int H, int W, int win_size, int sparsity,
                              int recon_scale, void *workspace, size_t workspace_bytes,
                              cudaStream_t stream)
{
    return cross_regression_impl("cross_regression", imga, imgb, albedo, normal, outa, outb, vara, varb, B, H, W,
                                 win_size, sparsity, recon_scale, 0.f, nullptr, workspace, workspace_bytes, stream);
}

cd_status cd_cross_regression_fp64_fallback(const float *imga, const float *imgb, const float *albedo,
                                             const float *normal, float *outa, float *outb, float *vara,
                                             float *varb, int B, int H, int W, int win_size, int sparsity,
                                             int recon_scale, float cond_limit, unsigned int *fallback_count,
                                             void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    if (!(cond_limit > 0.f)) {
        g_err[0] = 0;
        return fail(CD_EINVAL, "cross_regression_fp64_fallback: cond_limit must be > 0");
    }
    return cross_regression_impl("cross_regression_fp64_fallback", imga, imgb, albedo, normal, outa, outb, vara,
                                 varb, B, H, W, win_size, sparsity, recon_scale, cond_limit, fallback_count,
                                 workspace, workspace_bytes, stream);
}

size_t cd_cross_regression_grad_workspace_size(int B, int H, int W, int sparsity, int recon_scale)
{
    if (!dims_ok(B, H, W) || sparsity < 1 || recon_scale < 1) return 0;
    return cd::regression_grad_workspace_floats(B, H, W, sparsity, recon_scale) * sizeof(float);
}

cd_status cd_cross_regression_grad(const float *imga, const float *imgb, const float *albedo,
                                   const float *normal, const float *grad_outa, const float *grad_outb,
                                   const float *grad_vara, const float *grad_varb, float *grad_imga,
                                   float *grad_imgb, float *grad_albedo, float *grad_normal, int B, int H,
                                   int W, int win_size, int sparsity, int recon_scale, void *workspace,
                                   size_t workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!imga || !imgb || !albedo || !normal || !grad_outa || !grad_outb || !grad_imga || !grad_imgb ||
        !grad_albedo || !grad_normal)
        return fail(CD_EINVAL, "cross_regression_grad: null tensor pointer");
    cd_status s = check_regression("cross_regression_grad", B, H, W, win_size, sparsity, recon_scale);
    if (s != CD_OK) return s;
    const size_t need = cd_cross_regression_grad_workspace_size(B, H, W, sparsity, recon_scale);
    if (workspace_bytes < need || !workspace)
        return fail(CD_ENOMEM, "cross_regression_grad: workspace of %zu bytes needed, %zu given", need,
                    workspace_bytes);
    return cuda_status(cd::launch_regression_grad(imga, imgb, albedo, normal, grad_outa, grad_outb, grad_vara,
                                                  grad_varb, grad_imga, grad_imgb, grad_albedo, grad_normal, B, H,
                                                  W, win_size, sparsity, recon_scale,
                                                  static_cast<float *>(workspace), stream),
                       "cross_regression_grad");
}

cd_status cd_cross_regression_keep(const float *imga, const float *imgb, const float *albedo, const float *normal,
                                   float *outa, float *outb, float *vara, float *varb, int B, int H, int W,
                                   int win_size, int sparsity, int recon_scale, void *grad_workspace,
                                   size_t grad_workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!imga || !imgb || !albedo || !normal || !outa || !outb || !vara || !varb)
        return fail(CD_EINVAL, "cross_regression_keep: null tensor pointer");
    cd_status s = check_regression("cross_regression_keep", B, H, W, win_size, sparsity, recon_scale);
    if (s != CD_OK) return s;
    const size_t need = cd_cross_regression_grad_workspace_size(B, H, W, sparsity, recon_scale);
    if (grad_workspace_bytes < need || !grad_workspace)
        return fail(CD_ENOMEM, "cross_regression_keep: workspace of %zu bytes needed, %zu given", need,
                    grad_workspace_bytes);
    return cuda_status(cd::launch_regression_keep(imga, imgb, albedo, normal, outa, outb, vara, varb, B, H, W,
                                                  win_size, sparsity, recon_scale,
                                                  static_cast<float *>(grad_workspace), stream),
                       "cross_regression_keep");
}

cd_status cd_cross_regression_grad_kept(const float *imga, const float *imgb, const float *albedo,
                                        const float *normal, const float *grad_outa, const float *grad_outb,
                                        const float *grad_vara, const float *grad_varb, float *grad_imga,
                                        float *grad_imgb, float *grad_albedo, float *grad_normal, int B, int H,
                                        int W, int win_size, int sparsity, int recon_scale, void *grad_workspace,
                                        size_t grad_workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!imga || !imgb || !albedo || !normal || !grad_outa || !grad_outb || !grad_imga || !grad_imgb ||
        !grad_albedo || !grad_normal)
        return fail(CD_EINVAL, "cross_regression_grad_kept: null tensor pointer");
    cd_status s = check_regression("cross_regression_grad_kept", B, H, W, win_size, sparsity, recon_scale);
    if (s != CD_OK) return s;
    const size_t need = cd_cross_regression_grad_workspace_size(B, H, W, sparsity, recon_scale);
    if (grad_workspace_bytes < need || !grad_workspace)
        return fail(CD_ENOMEM, "cross_regression_grad_kept: workspace of %zu bytes needed, %zu given", need,
                    grad_workspace_bytes);
    return cuda_status(cd::launch_regression_grad(imga, imgb, albedo, normal, grad_outa, grad_outb, grad_vara,
                                                  grad_varb, grad_imga, grad_imgb, grad_albedo, grad_normal, B, H,
                                                  W, win_size, sparsity, recon_scale,
                                                  static_cast<float *>(grad_workspace), stream, true),
                       "cross_regression_grad_kept");
}

cd_status cd_spatial_filter(const float *imga, const float *imgb, const float *albedo,
                            const float *normal, const float *band, float *out_acca,
                            float *out_accb, float *out_wgtsuma, float *out_wgtsumb, int B, int H,
                            int W, int win_size, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!imga || !imgb || !albedo || !normal || !band || !out_acca || !out_accb || !out_wgtsuma || !out_wgtsumb)
        return fail(CD_EINVAL, "spatial_filter: null tensor pointer");
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "spatial_filter: bad shape B=%d H=%d W=%d", B, H, W);
    if (win_size < 1) return fail(CD_EINVAL, "spatial_filter: win_size must be >= 1");
    const int hw = win_size / 2;
    if (hw >= H || hw >= W)
        return fail(CD_EINVAL, "spatial_filter: window radius %d must be smaller than the image (%dx%d)", hw, H, W);
    if (cd::spatial_filter_smem_bytes(win_size) > kSmemLimit)
        return fail(CD_EINVAL, "spatial_filter: win_size %d exceeds the shared-memory tile", win_size);
    return cuda_status(cd::launch_spatial_filter(imga, imgb, albedo, normal, band, out_acca, out_accb,
                                                 out_wgtsuma, out_wgtsumb, B, H, W, win_size, stream),
                       "spatial_filter");
}

cd_status cd_spatial_filter_stored(const float *imga, const float *imgb, const float *albedo, const float *normal,
                                   const float *band, float *out_acca, float *out_accb, float *out_wgtsuma,
                                   float *out_wgtsumb, float *partials, int B, int H, int W, int win_size,
                                   cudaStream_t stream)
{
    g_err[0] = 0;
    if (!imga || !imgb || !albedo || !normal || !band || !out_acca || !out_accb || !out_wgtsuma || !out_wgtsumb ||
        !partials)
        return fail(CD_EINVAL, "spatial_filter_stored: null tensor pointer");
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "spatial_filter_stored: bad shape B=%d H=%d W=%d", B, H, W);
    if (win_size < 1) return fail(CD_EINVAL, "spatial_filter_stored: win_size must be >= 1");
    const int hw = win_size / 2;
    if (hw >= H || hw >= W)
        return fail(CD_EINVAL, "spatial_filter_stored: window radius %d must be smaller than the image (%dx%d)", hw,
                    H, W);
    if (cd::spatial_filter_smem_bytes(win_size) > kSmemLimit)
        return fail(CD_EINVAL, "spatial_filter_stored: win_size %d exceeds the shared-memory tile", win_size);
    return cuda_status(cd::launch_spatial_filter_store(imga, imgb, albedo, normal, band, out_acca, out_accb,
                                                       out_wgtsuma, out_wgtsumb, partials, B, H, W, win_size,
                                                       stream),
                       "spatial_filter_stored");
}

cd_status cd_spatial_filter_grad_stored(const float *grad_acca, const float *grad_accb, const float *grad_wgtsuma,
                                        const float *grad_wgtsumb, const float *partials, float *out_grad_band,
                                        int B, int H, int W, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!grad_acca || !grad_accb || !grad_wgtsuma || !grad_wgtsumb || !partials || !out_grad_band)
        return fail(CD_EINVAL, "spatial_filter_grad_stored: null tensor pointer");
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "spatial_filter_grad_stored: bad shape B=%d H=%d W=%d", B, H, W);
    return cuda_status(cd::launch_spatial_filter_grad_stored(grad_acca, grad_accb, grad_wgtsuma, grad_wgtsumb,
                                                             partials, out_grad_band, B, H, W, stream),
                       "spatial_filter_grad_stored");
}

cd_status cd_spatial_filter_grad(const float *grad_acca, const float *grad_accb,
                                 const float *grad_wgtsuma, const float *grad_wgtsumb,
                                 const float *imga, const float *imgb, const float *albedo,
                                 const float *normal, const float *band, float *out_grad_band,
                                 int B, int H, int W, int win_size, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!grad_acca || !grad_accb || !grad_wgtsuma || !grad_wgtsumb || !imga || !imgb || !albedo ||
        !normal || !band || !out_grad_band)
        return fail(CD_EINVAL, "spatial_filter_grad: null tensor pointer");
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "spatial_filter_grad: bad shape B=%d H=%d W=%d", B, H, W);
    if (win_size < 1) return fail(CD_EINVAL, "spatial_filter_grad: win_size must be >= 1");
    const int hw = win_size / 2;
    if (hw >= H || hw >= W)
        return fail(CD_EINVAL, "spatial_filter_grad: window radius %d must be smaller than the image (%dx%d)", hw, H, W);
    if (cd::spatial_filter_smem_bytes(win_size) > kSmemLimit)
        return fail(CD_EINVAL, "spatial_filter_grad: win_size %d exceeds the shared-memory tile", win_size);
    return cuda_status(cd::launch_spatial_filter_grad(grad_acca, grad_accb, grad_wgtsuma, grad_wgtsumb,
                                                      imga, imgb, albedo, normal, band, out_grad_band,
                                                      B, H, W, win_size, stream),
                       "spatial_filter_grad");
}

cd_status cd_reproject(const float *mvec, int n_list, const float *const *input_list,
                       const int *channels, float *const *output_list, const float *linear_z,
                       const float *prev_linear_z, const float *normal, const float *prev_normal,
                       const float *pn_fwidth, const float *opacity, const float *prev_opacity,
                       uint8_t *success, int B, int H, int W, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!mvec || !linear_z || !prev_linear_z || !normal || !prev_normal || !pn_fwidth || !opacity ||
        !prev_opacity || !success)
        return fail(CD_EINVAL, "reproject: null tensor pointer");
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "reproject: bad shape B=%d H=%d W=%d", B, H, W);
    if (n_list < 1 || n_list > CD_REPROJECT_MAX_LIST || !input_list || !output_list || !channels)
        return fail(CD_EINVAL, "reproject: input_list must hold 1..%d tensors", CD_REPROJECT_MAX_LIST);
    cd::ReprojectList list{};
    list.n = n_list;
    for (int d = 0; d < n_list; ++d) {
        if (!input_list[d] || !output_list[d])
            return fail(CD_EINVAL, "reproject: null pointer in input_list/output_list[%d]", d);
        if (channels[d] < 1 || channels[d] > 4096)
            return fail(CD_EINVAL, "reproject: input_list[%d] has %d channels", d, channels[d]);
        list.in[d] = input_list[d];
        list.out[d] = output_list[d];
        list.ch[d] = channels[d];
    }
    return cuda_status(cd::launch_reproject(mvec, list, linear_z, prev_linear_z, normal, prev_normal,
                                            pn_fwidth, opacity, prev_opacity, success, B, H, W, stream),
                       "reproject");
}

cd_status cd_erode3x3(const uint8_t *success, float *out, int B, int H, int W, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!success || !out) return fail(CD_EINVAL, "erode3x3: null tensor pointer");
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "erode3x3: bad shape B=%d H=%d W=%d", B, H, W);
    return cuda_status(cd::launch_erode3x3(success, out, B, H, W, stream), "erode3x3");
}

static cd_status temporal_checks(const char *name, int B, int H, int W, int win_curr, int win_prev)
{
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "%s: bad shape B=%d H=%d W=%d", name, B, H, W);
    if (win_curr < 1 || win_prev < 1) return fail(CD_EINVAL, "%s: win_curr and win_prev must be >= 1", name);
    if (temporal_tile_bytes(win_curr / 2) > kSmemLimit)
        return fail(CD_EINVAL, "%s: win_curr %d exceeds the shared-memory tile", name, win_curr);
    return CD_OK;
}

cd_status cd_temporal_screening(const float *current1, const float *current2, const float *prev,
                                const float *prev1, const float *prev2, const float *reproj_success,
                                float *output, float *output1, float *output2, float *success,
                                int B, int H, int W, int win_curr, int win_prev, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!current1 || !current2 || !prev || !prev1 || !prev2 || !reproj_success || !output || !output1 ||
        !output2 || !success)
        return fail(CD_EINVAL, "temporal_screening: null tensor pointer");
    cd_status s = temporal_checks("temporal_screening", B, H, W, win_curr, win_prev);
    if (s != CD_OK) return s;
    return cuda_status(cd::launch_temporal(current1, current2, prev, prev1, prev2, reproj_success, nullptr,
                                           nullptr, output, output1, output2, success, B, H, W, win_curr,
                                           win_prev, stream),
                       "temporal_screening");
}

cd_status cd_erode_temporal_screening(const float *current1, const float *current2, const float *prev,
                                      const float *prev1, const float *prev2, const uint8_t *reproj_mask,
                                      float *eroded, float *output, float *output1, float *output2,
                                      float *success, int B, int H, int W, int win_curr, int win_prev,
                                      cudaStream_t stream)
{
    g_err[0] = 0;
    if (!current1 || !current2 || !prev || !prev1 || !prev2 || !reproj_mask || !eroded || !output ||
        !output1 || !output2 || !success)
        return fail(CD_EINVAL, "erode_temporal_screening: null tensor pointer");
    cd_status s = temporal_checks("erode_temporal_screening", B, H, W, win_curr, win_prev);
    if (s != CD_OK) return s;
    return cuda_status(cd::launch_temporal(current1, current2, prev, prev1, prev2, nullptr, reproj_mask,
                                           eroded, output, output1, output2, success, B, H, W, win_curr,
                                           win_prev, stream),
                       "erode_temporal_screening");
}

cd_status cd_prepare_input(const float *color, const float *color2, float *y1, float *y2, size_t n,
                           cudaStream_t stream)
{
    g_err[0] = 0;
    if (!color || !color2 || !y1 || !y2) return fail(CD_EINVAL, "prepare_input: null tensor pointer");
    if (n == 0) return CD_OK;
    return cuda_status(cd::launch_log1p(color, color2, y1, y2, n, stream), "prepare_input");
}

size_t cd_aggregation_workspace_size(int B, int H, int W)
{
    if (!dims_ok(B, H, W)) return 0;
    return cd::aggregation_partials(B, H, W) * sizeof(float);
}

cd_status cd_aggregation_loss(const float *sum1, const float *sumw1, const float *sum2, const float *sumw2,
                              const float *alpha, const float *success, const float *success_prev,
                              const float *prev_out, const float *opacity, const float *label1,
                              const float *label2, const float *prev_label1, const float *prev_label2,
                              float *out_log, float *out, float *loss, float *avg_loss, float *grad_sum1,
                              float *grad_sumw1, float *grad_sum2, float *grad_sumw2, float *grad_alpha,
                              int B, int H, int W, void *workspace, size_t workspace_bytes,
                              cudaStream_t stream)
{
    g_err[0] = 0;
    if (!sum1 || !sumw1 || !sum2 || !sumw2 || !alpha || !success || !success_prev || !prev_out || !opacity ||
        !label1 || !label2 || !prev_label1 || !prev_label2 || !out_log || !out || !avg_loss || !grad_sum1 ||
        !grad_sumw1 || !grad_sum2 || !grad_sumw2 || !grad_alpha)
        return fail(CD_EINVAL, "aggregation_loss: null tensor pointer");
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "aggregation_loss: bad shape B=%d H=%d W=%d", B, H, W);
    const size_t need = cd_aggregation_workspace_size(B, H, W);
    if (workspace_bytes < need || !workspace)
        return fail(CD_ENOMEM, "aggregation_loss: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    cd::AggArgs A{sum1, sumw1, sum2, sumw2, alpha, success, success_prev, prev_out, opacity, label1, label2,
                  prev_label1, prev_label2, out_log, out, loss, grad_sum1, grad_sumw1, grad_sum2, grad_sumw2,
                  grad_alpha};
    return cuda_status(cd::launch_aggregation(A, static_cast<float *>(workspace), avg_loss, B, H, W, stream),
                       "aggregation_loss");
}

size_t cd_filter_aggregate_workspace_size(int B, int H, int W) { return cd_aggregation_workspace_size(B, H, W); }

cd_status cd_filter_aggregate(const float *ols1, const float *ols2, const float *albedo, const float *normal,
                              const float *band, const float *alpha, const float *success,
                              const float *success_prev, const float *prev_out, const float *opacity,
                              const float *prev_ols1, const float *prev_ols2, float *out_log, float *out,
                              float *avg_loss, float *grad_band, float *grad_alpha, int B, int H, int W,
                              int win_size, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!ols1 || !ols2 || !albedo || !normal || !band || !alpha || !success || !success_prev || !prev_out ||
        !opacity || !prev_ols1 || !prev_ols2 || !out_log || !out || !avg_loss || !grad_band || !grad_alpha)
        return fail(CD_EINVAL, "filter_aggregate: null tensor pointer");
    if (!dims_ok(B, H, W)) return fail(CD_EINVAL, "filter_aggregate: bad shape B=%d H=%d W=%d", B, H, W);
    if (win_size < 1) return fail(CD_EINVAL, "filter_aggregate: win_size must be >= 1");
    const int hw = win_size / 2;
    if (hw >= H || hw >= W)
        return fail(CD_EINVAL, "filter_aggregate: window radius %d must be smaller than the image (%dx%d)", hw, H, W);
    if (cd::filter_aggregate_smem(win_size) > kSmemLimit)
        return fail(CD_EINVAL, "filter_aggregate: win_size %d exceeds the shared-memory tile", win_size);
    const size_t need = cd_filter_aggregate_workspace_size(B, H, W);
    if (workspace_bytes < need || !workspace)
        return fail(CD_ENOMEM, "filter_aggregate: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    cd::AggArgs A{nullptr, nullptr, nullptr, nullptr, alpha, success, success_prev, prev_out, opacity, nullptr,
                  nullptr, prev_ols2, prev_ols1, out_log, out, nullptr, nullptr, nullptr, nullptr, nullptr,
                  grad_alpha};
    return cuda_status(cd::launch_filter_aggregate(ols1, ols2, albedo, normal, band, A, grad_band,
                                                   static_cast<float *>(workspace), avg_loss, B, H, W, win_size,
                                                   stream),
                       "filter_aggregate");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// U-Net kernel predictor and Adam
// ---------------------------------------------------------------------------
static bool unet_dims_ok(int B, int H, int W)
{
    return dims_ok(B, H, W) && H % 4 == 0 && W % 4 == 0 && H <= 4 * 65535;
}

// the tensor-core kernels stage activations and weights with bulk copies
static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

size_t cd_unet_param_count(void) { return (size_t)cd::unet::param_count(); }

size_t cd_unet_workspace_size(int B, int H, int W)
{
    return unet_dims_ok(B, H, W) ? cd::unet::workspace_bytes(B, H, W) : 0;
}

cd_status cd_unet_forward(const float *ols1, const float *ols2, const float *prev_out, const float *albedo,
                          const float *normal, const float *params, float *band, float *alpha, int B, int H, int W,
                          void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!ols1 || !ols2 || !prev_out || !albedo || !normal || !params || !band || !alpha)
        return fail(CD_EINVAL, "unet_forward: null pointer");
    if (!unet_dims_ok(B, H, W))
        return fail(CD_EINVAL, "unet_forward: bad shape B=%d H=%d W=%d (H and W must be multiples of 4)", B, H, W);
    const size_t need = cd::unet::workspace_bytes(B, H, W);
    if (!workspace || workspace_bytes < need)
        return fail(CD_ENOMEM, "unet_forward: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    if (!aligned16(workspace)) return fail(CD_EINVAL, "unet_forward: workspace not 16-byte aligned");
    return cuda_status(cd::unet::forward(ols1, ols2, prev_out, albedo, normal, params, band, alpha, workspace, B, H,
                                         W, stream),
                       "unet_forward");
}

cd_status cd_unet_backward(const float *grad_band, const float *grad_alpha, const float *params, float *grad_params,
                           int B, int H, int W, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!grad_band || !grad_alpha || !params || !grad_params) return fail(CD_EINVAL, "unet_backward: null pointer");
    if (!unet_dims_ok(B, H, W))
        return fail(CD_EINVAL, "unet_backward: bad shape B=%d H=%d W=%d (H and W must be multiples of 4)", B, H, W);
    const size_t need = cd::unet::workspace_bytes(B, H, W);
    if (!workspace || workspace_bytes < need)
        return fail(CD_ENOMEM, "unet_backward: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    if (!aligned16(workspace)) return fail(CD_EINVAL, "unet_backward: workspace not 16-byte aligned");
    return cuda_status(cd::unet::backward(grad_band, grad_alpha, params, grad_params, workspace, B, H, W, stream),
                       "unet_backward");
}

cd_status cd_adam_update(float *params, const float *grads, float *m, float *v, int n, int *step, float lr,
                         float beta1, float beta2, float epsilon, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!params || !grads || !m || !v || !step) return fail(CD_EINVAL, "adam_update: null pointer");
    if (n < 1) return fail(CD_EINVAL, "adam_update: n must be >= 1 (n=%d)", n);
    return cuda_status(cd::unet::adam(params, grads, m, v, n, step, lr, beta1, beta2, epsilon, stream), "adam_update");
}

static bool conv_channels_ok(int cin, int cout)
{
    const bool ci = cin == 8 || cin == 15 || cin == 16 || cin == 24 || cin == 32 || cin == 48;
    const bool co = cout == 8 || cout == 16 || cout == 32;
    return ci && co;
}

size_t cd_unet_conv3x3_workspace_size(int cin, int cout)
{
    return conv_channels_ok(cin, cout) ? cd::unet::conv_layer_workspace(cin, cout) : 0;
}

cd_status cd_unet_conv3x3(const float *weight, const float *bias, const void *x, void *y, int cin, int cout,
                          int dgrad, int B, int H, int W, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!weight || !x || !y || (!dgrad && !bias)) return fail(CD_EINVAL, "unet_conv3x3: null pointer");
    if (!conv_channels_ok(cin, cout)) return fail(CD_EINVAL, "unet_conv3x3: unsupported channels %d -> %d", cin, cout);
    if (!aligned16(x) || !aligned16(y) || !aligned16(workspace))
        return fail(CD_EINVAL, "unet_conv3x3: x, y and the workspace must be 16-byte aligned");
    if (!dims_ok(B, H, W) || H > 4 * 65535) return fail(CD_EINVAL, "unet_conv3x3: bad shape B=%d H=%d W=%d", B, H, W);
    const size_t need = cd::unet::conv_layer_workspace(cin, cout);
    if (!workspace || workspace_bytes < need)
        return fail(CD_ENOMEM, "unet_conv3x3: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    return cuda_status(cd::unet::conv_layer(weight, bias, static_cast<const __nv_bfloat16 *>(x),
                                            static_cast<__nv_bfloat16 *>(y), cin, cout, dgrad ? 1 : 0, B, H, W,
                                            workspace, stream),
                       "unet_conv3x3");
}

size_t cd_unet_conv3x3_wgrad_workspace_size(int cin, int cout, int B, int H, int W)
{
    return conv_channels_ok(cin, cout) && dims_ok(B, H, W) ? cd::unet::wgrad_layer_workspace(cin, cout, B, H, W) : 0;
}

cd_status cd_unet_conv3x3_wgrad(const void *x, const void *dz, float *grad, int cin, int cout, int B, int H, int W,
                                void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    g_err[0] = 0;
    if (!x || !dz || !grad) return fail(CD_EINVAL, "unet_conv3x3_wgrad: null pointer");
    if (!conv_channels_ok(cin, cout))
        return fail(CD_EINVAL, "unet_conv3x3_wgrad: unsupported channels %d -> %d", cin, cout);
    if (!aligned16(x) || !aligned16(dz)) return fail(CD_EINVAL, "unet_conv3x3_wgrad: x and dz must be 16-byte aligned");
    if (!dims_ok(B, H, W) || H > 4 * 65535)
        return fail(CD_EINVAL, "unet_conv3x3_wgrad: bad shape B=%d H=%d W=%d", B, H, W);
    const size_t need = cd::unet::wgrad_layer_workspace(cin, cout, B, H, W);
    if (!workspace || workspace_bytes < need)
        return fail(CD_ENOMEM, "unet_conv3x3_wgrad: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    return cuda_status(cd::unet::wgrad_layer(static_cast<const __nv_bfloat16 *>(x),
                                             static_cast<const __nv_bfloat16 *>(dz), grad, cin, cout, B, H, W,
                                             workspace, stream),
                       "unet_conv3x3_wgrad");
}
