// Test infrastructure: compiles the reference's ops/temporal.cu.cc as it is
// (its TensorFlow wrapper half against the stand-in headers in shim/) and
// launches its TemporalScreening kernel (ops/temporal.cu.cc:57-198) with the
// wrapper's 8x8 launch shape (:238-255).
#include "temporal.cu.cc"

extern "C" int cdref_temporal_screening(const float *c1, const float *c2, const float *prev,
                                        const float *prev1, const float *prev2, const float *rs,
                                        float *out, float *out1, float *out2, float *succ, int H,
                                        int W, int win_curr, int win_prev, void *stream)
{
    dim3 threads(8, 8);
    dim3 grid(iDivUp(W, 8), iDivUp(H, 8));
    TemporalScreening<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        out, out1, out2, succ, c1, c2, prev, prev1, prev2, rs, H, W, win_curr, win_prev);
    return static_cast<int>(cudaGetLastError());
}
