// cd_cross_regression_noalloc: cross-regression for callers that cannot
// hand the library a workspace.
//
// Some hosts of this op cannot allocate device memory when it runs: a
// renderer's or game engine's frame loop that owns every device allocation
// through its own pool and forbids allocations mid-frame (a cudaMalloc can
// synchronise the device and stall the frame, or fail under memory pressure
// at the worst moment), and plugin hosts that pass tensors in but expose no
// allocator to their plugins.  For them the coefficients and standard
// deviations that cd_cross_regression keeps in its workspace live here, in
// one file-scope device array that the driver allocates when the library's
// module is loaded on a device and that stays allocated until the process
// exits.  Nothing in this file calls cudaMalloc or cudaFree.
//
// Limits and sharing, as documented in include/cd_ops.h:
//   * the array holds kNoAllocBytes; larger problems are rejected;
//   * every call on a device uses the same array, so calls whose kernels
//     overlap on the GPU (different streams, or host threads racing) corrupt
//     each other -- serialise them;
//   * the first call on each device resolves the array's device address
//     (cudaGetSymbolAddress) and caches it; make that first call before any
//     stream capture.  The cache is not invalidated by cudaDeviceReset, so a
//     process that resets a device must not call this entry point on it
//     afterwards.
// Nothing in the array has to start at zero: the variance kernel writes
// every standard deviation and the regression kernel every coefficient
// before the reconstruction reads them.
#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>
#include "cd_common.cuh"
#include "../../include/cd_ops.h"

namespace {

constexpr size_t kNoAllocBytes = (size_t)CD_NOALLOC_SCRATCH_MIB << 20;

__device__ __align__(256) unsigned char g_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device (resolved once per device).
cudaError_t scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" size_t cd_cross_regression_noalloc_capacity(void) { return kNoAllocBytes; }

extern "C" cd_status cd_cross_regression_noalloc(const float *imga, const float *imgb, const float *albedo,
                                                 const float *normal, float *outa, float *outb, float *vara,
                                                 float *varb, int B, int H, int W, int win_size, int sparsity,
                                                 int recon_scale, cudaStream_t stream)
{
    // Invalid arguments are reported as the regular entry point reports
    // them (CD_EINVAL), before the size check; a valid problem must then fit
    // the static array.
    cd::set_last_error("");
    const int bad = cd::check_cross_regression_args("cross_regression_noalloc", imga, imgb, albedo, normal, outa,
                                                    outb, vara, varb, B, H, W, win_size, sparsity, recon_scale);
    if (bad != CD_OK) return static_cast<cd_status>(bad);
    const size_t need = cd_cross_regression_workspace_size(B, H, W, sparsity);
    if (need > kNoAllocBytes) {
        char g_msg[256];
        snprintf(g_msg, sizeof(g_msg),
                 "cross_regression_noalloc: needs %zu bytes of scratch, the built-in array holds %zu "
                 "(%d MiB); use cd_cross_regression with a workspace", need, kNoAllocBytes,
                 (int)CD_NOALLOC_SCRATCH_MIB);
        cd::set_last_error(g_msg);
        return CD_ENOMEM;
    }
    void *scratch = nullptr;
    const cudaError_t e = scratch_address(&scratch);
    if (e != cudaSuccess) {
        char g_msg[256];
        snprintf(g_msg, sizeof(g_msg), "cross_regression_noalloc: cudaGetSymbolAddress failed: %s",
                 cudaGetErrorString(e));
        cd::set_last_error(g_msg);
        return CD_ECUDA;
    }
    return cd_cross_regression(imga, imgb, albedo, normal, outa, outb, vara, varb, B, H, W, win_size, sparsity,
                               recon_scale, scratch, kNoAllocBytes, stream);
}
