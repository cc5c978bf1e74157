// Cross-bilateral spatial filter on sm_100a, forward and band gradient.
//
// Reference semantics: SpatialFilterKernel and SpatialFilterGradKernel,
// ops/regression.cu.cc:33-195.  For every pixel p and every tap t of the
// win x win reflect-101 window:
//   e_A = -band0*|A_p-A_t|^2 - band2*|alb_p-alb_t|^2 - band3*|n_p-n_t|^2 - band4*d(p,t)
//   e_B = the same with band1 and image B,  d = ((dx/r)^2 + (dy/r)^2), r = win/2
//   acc_A += exp(e_A) * A_t,  wsum_A += exp(e_A)   (and B likewise)
// The reference forward also stores 128 B/px of d(acc, wsum)/d(band) partials
// for its gradient op; here the gradient kernel recomputes the weights and
// the partials in registers and dots them with the upstream gradient:
//   dL/dband_k(p) = g_acc(p) . P_k(p) + g_wsum(p) P_k.w(p),
//   P_k(p) = sum_t exp(e)(-dist_k) [col_t, 1],
// with channel 0 from A only, 1 from B only and 2..4 from A + B.
//
// Both kernels stage the CTA's footprint (32x8 pixels plus the window radius)
// in shared memory and run the packed A/B window sweep of filter_sweep.cuh;
// radii 3, 5 and 7 (windows 7, 11, 15) are compiled with the window loop
// unrolled, other radii take the radius at run time.
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "filter_sweep.cuh"

namespace cd {
namespace {

using fsw::f2;

template <int HW>
__global__ void __launch_bounds__(256) sf_forward_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ band, float *__restrict__ acca, float *__restrict__ accb,
    float *__restrict__ wsa, float *__restrict__ wsb, int H, int W, int hw_rt)
{
    extern __shared__ ulonglong2 tile[];
    const int hw = HW > 0 ? HW : hw_rt;
    const int tw = fsw::kBX + 2 * hw, th = fsw::kBY + 2 * hw;
    f2 *pdtab = reinterpret_cast<f2 *>(tile + 3 * tw * th);
    const size_t px = (size_t)H * W, b = blockIdx.z;
    fsw::stage(tile, pdtab, imga + 3 * px * b, imgb + 3 * px * b, albedo + 3 * px * b, normal + 3 * px * b,
               H, W, hw);
    __syncthreads();
    const int cx = blockIdx.x * fsw::kBX + threadIdx.x, cy = blockIdx.y * fsw::kBY + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const size_t p = b * px + (size_t)cy * W + cx;
    const fsw::Centre c = fsw::centre(tile, hw, band + 5 * p);
    fsw::Sums s;
    fsw::zero(s);
    fsw::sweep<HW, true, false>(tile, pdtab, hw, c, s);
    st3(acca, p, make_float3(fsw::lo(s.acc_x), fsw::lo(s.acc_y), fsw::lo(s.acc_z)));
    st3(accb, p, make_float3(fsw::hi(s.acc_x), fsw::hi(s.acc_y), fsw::hi(s.acc_z)));
    wsa[p] = fsw::lo(s.acc_w);
    wsb[p] = fsw::hi(s.acc_w);
}

template <int HW>
__global__ void __launch_bounds__(256, 3) sf_grad_kernel(
    const float *__restrict__ gacca, const float *__restrict__ gaccb,
    const float *__restrict__ gwsa, const float *__restrict__ gwsb,
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ band, float *__restrict__ gband, int H, int W, int hw_rt)
{
    extern __shared__ ulonglong2 tile[];
    const int hw = HW > 0 ? HW : hw_rt;
    const int tw = fsw::kBX + 2 * hw, th = fsw::kBY + 2 * hw;
    f2 *pdtab = reinterpret_cast<f2 *>(tile + 3 * tw * th);
    const size_t px = (size_t)H * W, b = blockIdx.z;
    fsw::stage(tile, pdtab, imga + 3 * px * b, imgb + 3 * px * b, albedo + 3 * px * b, normal + 3 * px * b,
               H, W, hw);
    __syncthreads();
    const int cx = blockIdx.x * fsw::kBX + threadIdx.x, cy = blockIdx.y * fsw::kBY + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const size_t p = b * px + (size_t)cy * W + cx;
    const fsw::Centre c = fsw::centre(tile, hw, band + 5 * p);
    fsw::Sums s;
    fsw::zero(s);
    // the reference's per-pixel band partials (ops/regression.cu.cc:157-177),
    // accumulated in registers and dotted with the upstream gradient as
    // SpatialFilterGradKernel does (:64-80)
    fsw::sweep<HW, false, true>(tile, pdtab, hw, c, s);
    fsw::band_grad(s, ld3(gacca, p), ld3(gaccb, p), __ldg(gwsa + p), __ldg(gwsb + p), gband + 5 * p);
}

// Stored-partials variant, the reference's design (its forward keeps 128 B
// per pixel of band partials for the gradient op): the forward also writes
// P[p] = {A: P_0..P_3, B: P_0..P_3} x (col.xyz, 1), 32 floats per pixel, and
// the gradient kernel only reads them.  Kept for the recompute-vs-store
// measurement; the sums are the recomputing kernels' to the bit.
template <int HW>
__global__ void __launch_bounds__(256) sf_forward_store_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ band, float *__restrict__ acca, float *__restrict__ accb,
    float *__restrict__ wsa, float *__restrict__ wsb, float4 *__restrict__ part, int H, int W, int hw_rt)
{
    extern __shared__ ulonglong2 tile[];
    const int hw = HW > 0 ? HW : hw_rt;
    const int tw = fsw::kBX + 2 * hw, th = fsw::kBY + 2 * hw;
    f2 *pdtab = reinterpret_cast<f2 *>(tile + 3 * tw * th);
    const size_t px = (size_t)H * W, b = blockIdx.z;
    fsw::stage(tile, pdtab, imga + 3 * px * b, imgb + 3 * px * b, albedo + 3 * px * b, normal + 3 * px * b,
               H, W, hw);
    __syncthreads();
    const int cx = blockIdx.x * fsw::kBX + threadIdx.x, cy = blockIdx.y * fsw::kBY + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const size_t p = b * px + (size_t)cy * W + cx;
    const fsw::Centre c = fsw::centre(tile, hw, band + 5 * p);
    fsw::Sums s;
    fsw::zero(s);
    fsw::sweep<HW, true, true>(tile, pdtab, hw, c, s);
    st3(acca, p, make_float3(fsw::lo(s.acc_x), fsw::lo(s.acc_y), fsw::lo(s.acc_z)));
    st3(accb, p, make_float3(fsw::hi(s.acc_x), fsw::hi(s.acc_y), fsw::hi(s.acc_z)));
    wsa[p] = fsw::lo(s.acc_w);
    wsb[p] = fsw::hi(s.acc_w);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        part[8 * p + k] = make_float4(fsw::lo(s.px[k]), fsw::lo(s.py[k]), fsw::lo(s.pz[k]), fsw::lo(s.pw[k]));
        part[8 * p + 4 + k] = make_float4(fsw::hi(s.px[k]), fsw::hi(s.py[k]), fsw::hi(s.pz[k]), fsw::hi(s.pw[k]));
    }
}

__global__ void __launch_bounds__(256) sf_grad_stored_kernel(const float *__restrict__ gacca,
                                                             const float *__restrict__ gaccb,
                                                             const float *__restrict__ gwsa,
                                                             const float *__restrict__ gwsb,
                                                             const float4 *__restrict__ part,
                                                             float *__restrict__ gband, size_t n)
{
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    fsw::Sums s;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 a = __ldg(part + 8 * p + k), bb = __ldg(part + 8 * p + 4 + k);
        s.px[k] = fsw::pack(a.x, bb.x);
        s.py[k] = fsw::pack(a.y, bb.y);
        s.pz[k] = fsw::pack(a.z, bb.z);
        s.pw[k] = fsw::pack(a.w, bb.w);
    }
    fsw::band_grad(s, ld3(gacca, p), ld3(gaccb, p), __ldg(gwsa + p), __ldg(gwsb + p), gband + 5 * p);
}

template <typename F>
cudaError_t dispatch_radius(int hw, F &&launch)
{
    switch (hw) {
    case 3: return launch(std::integral_constant<int, 3>());
    case 5: return launch(std::integral_constant<int, 5>());
    case 7: return launch(std::integral_constant<int, 7>());
    default: return launch(std::integral_constant<int, 0>());
    }
}

}  // namespace

size_t spatial_filter_smem_bytes(int win) { return fsw::smem_bytes(win / 2); }

cudaError_t launch_spatial_filter_store(const float *imga, const float *imgb, const float *albedo,
                                        const float *normal, const float *band, float *acca, float *accb,
                                        float *wsa, float *wsb, float *partials, int B, int H, int W, int win,
                                        cudaStream_t st)
{
    const int hw = win / 2;
    const size_t smem = fsw::smem_bytes(hw);
    dim3 grid((W + fsw::kBX - 1) / fsw::kBX, (H + fsw::kBY - 1) / fsw::kBY, B), block(fsw::kBX, fsw::kBY);
    return dispatch_radius(hw, [&](auto r) {
        constexpr int R = decltype(r)::value;
        cudaError_t e = cudaFuncSetAttribute(sf_forward_store_kernel<R>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        sf_forward_store_kernel<R><<<grid, block, smem, st>>>(imga, imgb, albedo, normal, band, acca, accb, wsa,
                                                              wsb, reinterpret_cast<float4 *>(partials), H, W, hw);
        return cudaGetLastError();
    });
}

cudaError_t launch_spatial_filter_grad_stored(const float *gacca, const float *gaccb, const float *gwsa,
                                              const float *gwsb, const float *partials, float *gband, int B, int H,
                                              int W, cudaStream_t st)
{
    const size_t n = (size_t)B * H * W;
    sf_grad_stored_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        gacca, gaccb, gwsa, gwsb, reinterpret_cast<const float4 *>(partials), gband, n);
    return cudaGetLastError();
}

cudaError_t launch_spatial_filter(const float *imga, const float *imgb, const float *albedo,
                                  const float *normal, const float *band, float *acca,
                                  float *accb, float *wsa, float *wsb, int B, int H, int W,
                                  int win, cudaStream_t st)
{
    const int hw = win / 2;
    const size_t smem = fsw::smem_bytes(hw);
    dim3 grid((W + fsw::kBX - 1) / fsw::kBX, (H + fsw::kBY - 1) / fsw::kBY, B), block(fsw::kBX, fsw::kBY);
    return dispatch_radius(hw, [&](auto r) {
        constexpr int R = decltype(r)::value;
        cudaError_t e = cudaFuncSetAttribute(sf_forward_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        sf_forward_kernel<R><<<grid, block, smem, st>>>(imga, imgb, albedo, normal, band, acca, accb, wsa, wsb,
                                                        H, W, hw);
        return cudaGetLastError();
    });
}

cudaError_t launch_spatial_filter_grad(const float *gacca, const float *gaccb, const float *gwsa,
                                       const float *gwsb, const float *imga, const float *imgb,
                                       const float *albedo, const float *normal,
                                       const float *band, float *gband, int B, int H, int W,
                                       int win, cudaStream_t st)
{
    const int hw = win / 2;
    const size_t smem = fsw::smem_bytes(hw);
    dim3 grid((W + fsw::kBX - 1) / fsw::kBX, (H + fsw::kBY - 1) / fsw::kBY, B), block(fsw::kBX, fsw::kBY);
    return dispatch_radius(hw, [&](auto r) {
        constexpr int R = decltype(r)::value;
        cudaError_t e = cudaFuncSetAttribute(sf_grad_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        sf_grad_kernel<R><<<grid, block, smem, st>>>(gacca, gaccb, gwsa, gwsb, imga, imgb, albedo, normal, band,
                                                     gband, H, W, hw);
        return cudaGetLastError();
    });
}

}  // namespace cd
