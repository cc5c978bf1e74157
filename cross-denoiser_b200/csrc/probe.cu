// FP32 FMA throughput probe: the denominator of the roofline of the FP32
// (non-tensor) kernels.  Every thread runs 8 independent FMA chains; the
// result is stored so the chains cannot be removed.  Not part of the
// reference's interface.
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "../../include/cd_ops.h"

namespace {
__global__ void __launch_bounds__(256) fma_probe_kernel(float *out, int iters, float a, float b)
{
    float x0 = threadIdx.x, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
}
}  // namespace

extern "C" cd_status cd_fp32_fma_probe(float *out, int blocks, int iters, cudaStream_t stream)
{
    if (!out || blocks < 1 || iters < 1) return CD_EINVAL;
    fma_probe_kernel<<<blocks, 256, 0, stream>>>(out, iters, 0.999999f, 1e-7f);
    return cudaGetLastError() == cudaSuccess ? CD_OK : CD_ECUDA;
}
