// Test infrastructure: compiles the reference's ops/reproject.cu.cc as it is
// and exposes ReprojectFunc (ops/reproject.cu.cc:240-273) through a C ABI.
// The wrapper repeats what ReprojectOp::Compute does around the launch
// (ops/reproject.cc:140-153): device-side dims / pointer tables allocated once
// and refreshed with blocking cudaMemcpy on every call.
#include "reproject.cu.cc"

static int *g_dims = nullptr;
static const float **g_inputs = nullptr;
static float **g_outputs = nullptr;
static const int kMaxList = 16;

extern "C" int cdref_reproject(const float *mvec, int n_list, const float *const *inputs,
                               const int *channels, float *const *outputs, const float *linz,
                               const float *plinz, const float *nrm, const float *pnrm,
                               const float *pnfw, const float *opac, const float *popac,
                               unsigned char *success, int B, int H, int W, void *stream)
{
    if (n_list < 1 || n_list > kMaxList) return -1;
    cudaError_t e;
    if (g_dims == nullptr) {
        if ((e = cudaMalloc((void **)&g_dims, sizeof(int) * kMaxList)) != cudaSuccess) return (int)e;
        if ((e = cudaMalloc((void **)&g_inputs, sizeof(float *) * kMaxList)) != cudaSuccess) return (int)e;
        if ((e = cudaMalloc((void **)&g_outputs, sizeof(float *) * kMaxList)) != cudaSuccess) return (int)e;
    }
    if ((e = cudaMemcpy(g_dims, channels, sizeof(int) * n_list, cudaMemcpyHostToDevice)) != cudaSuccess) return (int)e;
    if ((e = cudaMemcpy(g_inputs, inputs, sizeof(float *) * n_list, cudaMemcpyHostToDevice)) != cudaSuccess) return (int)e;
    if ((e = cudaMemcpy(g_outputs, outputs, sizeof(float *) * n_list, cudaMemcpyHostToDevice)) != cudaSuccess) return (int)e;
    Eigen::GpuDevice dev(static_cast<cudaStream_t>(stream));
    ReprojectFunc(dev, mvec, g_dims, g_inputs, linz, plinz, nrm, pnrm, pnfw, opac, popac, g_outputs,
                  reinterpret_cast<bool *>(success), B, n_list, H, W);
    return static_cast<int>(cudaGetLastError());
}
