// Test infrastructure: compiles the reference's ops/regression.cu.cc as it is
// (include path points at the reference tree) and exposes its launchers
// CrossRegressionFunc / SpatialFilterFunc / SpatialFilterGradFunc
// (ops/regression.cu.cc:477-534) through a C ABI, for the parity tests and
// the reference arm of bench.py.  The callers replicate the TF op wrappers'
// scratch handling (ops/regression.cc:138-145, 174-182, 209-225): the beta
// and band-partial buffers are allocated and zeroed once and then reused.
#include "regression.cu.cc"

extern "C" {

int cdref_cross_regression(const float *imga, const float *imgb, const float *albedo,
                           const float *normal, float *outa, float *outb, float *vara,
                           float *varb, float *betaA, float *betaB, int H, int W, int win,
                           int sparsity, int recon_scale, void *stream)
{
    Eigen::GpuDevice dev(static_cast<cudaStream_t>(stream));
    CrossRegressionFunc(dev, imga, imgb, albedo, normal, outa, outb, vara, varb,
                        reinterpret_cast<float4 *>(betaA), reinterpret_cast<float4 *>(betaB),
                        1, H, W, win, sparsity, recon_scale);
    return static_cast<int>(cudaGetLastError());
}

int cdref_spatial_filter(const float *imga, const float *imgb, const float *albedo,
                         const float *normal, const float *band, float *acca, float *accb,
                         float *wsa, float *wsb, float *partA, float *partB, int H, int W,
                         int win, void *stream)
{
    Eigen::GpuDevice dev(static_cast<cudaStream_t>(stream));
    SpatialFilterFunc(dev, imga, imgb, albedo, normal, band, acca, accb, wsa, wsb,
                      reinterpret_cast<float4 *>(partA), reinterpret_cast<float4 *>(partB),
                      1, H, W, win);
    return static_cast<int>(cudaGetLastError());
}

int cdref_spatial_filter_grad(const float *g_acca, const float *g_accb, const float *g_wsa,
                              const float *g_wsb, const float *imga, const float *imgb,
                              const float *albedo, const float *normal, const float *band,
                              float *gband, const float *partA, const float *partB, int H,
                              int W, int win, void *stream)
{
    Eigen::GpuDevice dev(static_cast<cudaStream_t>(stream));
    SpatialFilterGradFunc(dev, g_acca, g_accb, g_wsa, g_wsb, imga, imgb, albedo, normal, band,
                          gband, reinterpret_cast<const float4 *>(partA),
                          reinterpret_cast<const float4 *>(partB), 1, H, W, win);
    return static_cast<int>(cudaGetLastError());
}

}  // extern "C"
