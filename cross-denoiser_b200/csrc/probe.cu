// Probes behind the measurements and the error handling, not part of the
// reference's interface:
//   * FP32 FMA throughput: the denominator of the roofline of the FP32
//     (non-tensor) kernels.  Every thread runs 8 independent FMA chains; the
//     result is stored so the chains cannot be removed.
//   * the bounded mbarrier wait of the tensor-core kernels (tc::mbar_wait)
//     running out on a barrier that nothing arrives at, with no copy or MMA
//     in flight, and the error flag it sets.
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "tc_sm100.cuh"
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

// One warp: thread 0 initialises a one-arrival mbarrier and, if `arrive`,
// arrives on it; then the warp waits for phase 0 exactly as the tensor-core
// kernels wait for their copies and MMAs (uniform decision), and on time-out
// thread 0 sets *flag to 1 as they set their workspace flag.
__global__ void __launch_bounds__(32) mbar_timeout_kernel(int *flag, int arrive, int max_iter)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        cd::tc::mbar_init(&bar, 1);
        if (arrive) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(cd::tc::smem_u32(&bar)) : "memory");
    }
    __syncthreads();
    const bool ok = __syncthreads_and(cd::tc::mbar_wait(&bar, 0, max_iter)) != 0;
    if (!ok && threadIdx.x == 0) atomicExch(flag, 1);
}
}  // namespace

extern "C" cd_status cd_mbar_timeout_probe(int *flag, int arrive, int max_iter, cudaStream_t stream)
{
    if (!flag || max_iter < 1 || max_iter > CD_MBAR_PROBE_MAX_ITER) return CD_EINVAL;
    mbar_timeout_kernel<<<1, 32, 0, stream>>>(flag, arrive ? 1 : 0, max_iter);
    return cudaGetLastError() == cudaSuccess ? CD_OK : CD_ECUDA;
}

extern "C" cd_status cd_fp32_fma_probe(float *out, int blocks, int iters, cudaStream_t stream)
{
    if (!out || blocks < 1 || iters < 1) return CD_EINVAL;
    fma_probe_kernel<<<blocks, 256, 0, stream>>>(out, iters, 0.999999f, 1e-7f);
    return cudaGetLastError() == cudaSuccess ? CD_OK : CD_ECUDA;
}
