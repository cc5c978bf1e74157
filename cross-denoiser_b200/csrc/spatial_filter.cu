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
// in shared memory as 12 SoA planes (A.xyz, B.xyz, albedo.xyz, normal.xyz); a
// warp reads one tile row, so the loads are bank-conflict free.
#include <cuda_runtime.h>
#include "cd_common.cuh"

namespace cd {
namespace {

constexpr int kBX = 32, kBY = 8;
constexpr int kPlanes = 12;
constexpr int kMaxTable = 128;   // entries of the dx/r table (win <= 255)

__host__ __device__ inline size_t sf_smem(int hw)
{
    return (size_t)kPlanes * (kBX + 2 * hw) * (kBY + 2 * hw) * sizeof(float) +
           kMaxTable * 2 * sizeof(float);
}

struct Px {
    float a[3], b[3], al[3], n[3];
};

// Loads the footprint of this CTA into the planes and the (d/r) table.
CD_DEV void stage_tile(float *sm, float *tab, const float *imga, const float *imgb,
                       const float *albedo, const float *normal, int H, int W, int hw)
{
    const int tw = kBX + 2 * hw, th = kBY + 2 * hw;
    const int plane = tw * th;
    const int x0 = blockIdx.x * kBX - hw, y0 = blockIdx.y * kBY - hw;
    const int tid = threadIdx.y * kBX + threadIdx.x;
    for (int t = tid; t < plane; t += kBX * kBY) {
        const int ty = t / tw, tx = t - ty * tw;
        const int gx = min(max(mirror(x0 + tx, W), 0), W - 1);
        const int gy = min(max(mirror(y0 + ty, H), 0), H - 1);
        const size_t q = (size_t)gy * W + gx;
        const float3 a = ld3(imga, q), b = ld3(imgb, q), al = ld3(albedo, q), n = ld3(normal, q);
        sm[0 * plane + t] = a.x;
        sm[1 * plane + t] = a.y;
        sm[2 * plane + t] = a.z;
        sm[3 * plane + t] = b.x;
        sm[4 * plane + t] = b.y;
        sm[5 * plane + t] = b.z;
        sm[6 * plane + t] = al.x;
        sm[7 * plane + t] = al.y;
        sm[8 * plane + t] = al.z;
        sm[9 * plane + t] = n.x;
        sm[10 * plane + t] = n.y;
        sm[11 * plane + t] = n.z;
    }
    // tab[k] = (float)(hw - k) / hw, i.e. (c - i) / r for tap offset k - hw
    for (int k = tid; k <= 2 * hw; k += kBX * kBY) tab[k] = (float)(hw - k) / (float)hw;
}

CD_DEV Px load_px(const float *sm, int plane, int o)
{
    Px p;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p.a[k] = sm[k * plane + o];
        p.b[k] = sm[(3 + k) * plane + o];
        p.al[k] = sm[(6 + k) * plane + o];
        p.n[k] = sm[(9 + k) * plane + o];
    }
    return p;
}

CD_DEV float dist3(const float *c, const float *t)
{
    return norm2(c[0] - t[0], c[1] - t[1], c[2] - t[2]);
}

__global__ void __launch_bounds__(256) sf_forward_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ band, float *__restrict__ acca, float *__restrict__ accb,
    float *__restrict__ wsa, float *__restrict__ wsb, int H, int W, int hw)
{
    extern __shared__ float sm[];
    const int tw = kBX + 2 * hw, th = kBY + 2 * hw, plane = tw * th;
    float *tab = sm + kPlanes * plane;
    const size_t px = (size_t)H * W, b = blockIdx.z;
    imga += 3 * px * b;
    imgb += 3 * px * b;
    albedo += 3 * px * b;
    normal += 3 * px * b;
    stage_tile(sm, tab, imga, imgb, albedo, normal, H, W, hw);
    __syncthreads();

    const int cx = blockIdx.x * kBX + threadIdx.x, cy = blockIdx.y * kBY + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const size_t p = b * px + (size_t)cy * W + cx;
    const float b0 = __ldg(band + 5 * p), b1 = __ldg(band + 5 * p + 1), b2 = __ldg(band + 5 * p + 2);
    const float b3 = __ldg(band + 5 * p + 3), b4 = __ldg(band + 5 * p + 4);
    const Px c = load_px(sm, plane, (threadIdx.y + hw) * tw + threadIdx.x + hw);

    float aA[3] = {0.f, 0.f, 0.f}, aB[3] = {0.f, 0.f, 0.f}, sA = 0.f, sB = 0.f;
    for (int ky = 0; ky <= 2 * hw; ++ky) {
        const float dyf = tab[ky];
        const int rowo = (threadIdx.y + ky) * tw + threadIdx.x;
        for (int kx = 0; kx <= 2 * hw; ++kx) {
            const float dxf = tab[kx];
            const float pd = dxf * dxf + dyf * dyf;
            const Px t = load_px(sm, plane, rowo + kx);
            const float dA = dist3(c.a, t.a), dB = dist3(c.b, t.b);
            const float dAl = dist3(c.al, t.al), dN = dist3(c.n, t.n);
            const float eA = -b0 * dA - b2 * dAl - b3 * dN - b4 * pd;
            const float eB = -b1 * dB - b2 * dAl - b3 * dN - b4 * pd;
            const float wA = __expf(eA), wB = __expf(eB);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                aA[k] = fmaf(wA, t.a[k], aA[k]);
                aB[k] = fmaf(wB, t.b[k], aB[k]);
            }
            sA += wA;
            sB += wB;
        }
    }
    st3(acca, p, make_float3(aA[0], aA[1], aA[2]));
    st3(accb, p, make_float3(aB[0], aB[1], aB[2]));
    wsa[p] = sA;
    wsb[p] = sB;
}

__global__ void __launch_bounds__(256) sf_grad_kernel(
    const float *__restrict__ gacca, const float *__restrict__ gaccb,
    const float *__restrict__ gwsa, const float *__restrict__ gwsb,
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ band, float *__restrict__ gband, int H, int W, int hw)
{
    extern __shared__ float sm[];
    const int tw = kBX + 2 * hw, th = kBY + 2 * hw, plane = tw * th;
    float *tab = sm + kPlanes * plane;
    const size_t px = (size_t)H * W, b = blockIdx.z;
    imga += 3 * px * b;
    imgb += 3 * px * b;
    albedo += 3 * px * b;
    normal += 3 * px * b;
    stage_tile(sm, tab, imga, imgb, albedo, normal, H, W, hw);
    __syncthreads();

    const int cx = blockIdx.x * kBX + threadIdx.x, cy = blockIdx.y * kBY + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const size_t p = b * px + (size_t)cy * W + cx;
    const float b0 = __ldg(band + 5 * p), b1 = __ldg(band + 5 * p + 1), b2 = __ldg(band + 5 * p + 2);
    const float b3 = __ldg(band + 5 * p + 3), b4 = __ldg(band + 5 * p + 4);
    const float3 gA = ld3(gacca, p), gB = ld3(gaccb, p);
    const float gwA = __ldg(gwsa + p), gwB = __ldg(gwsb + p);
    const Px c = load_px(sm, plane, (threadIdx.y + hw) * tw + threadIdx.x + hw);

    // Per-pixel band partials d(acc, wsum)/d(band_k) = sum_t w_t (-dist_k)
    // [col_t, 1], accumulated tap by tap exactly as the reference forward
    // does (ops/regression.cu.cc:157-177), then dotted with the upstream
    // gradient as SpatialFilterGradKernel does (:64-80).  Keeping the
    // reference's association avoids the cancellation differences a folded
    // sum_t w (-dist_k)(g . col_t + g_w) would introduce.
    float4 pA[4], pB[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        pA[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        pB[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    for (int ky = 0; ky <= 2 * hw; ++ky) {
        const float dyf = tab[ky];
        const int rowo = (threadIdx.y + ky) * tw + threadIdx.x;
        for (int kx = 0; kx <= 2 * hw; ++kx) {
            const float dxf = tab[kx];
            const float pd = dxf * dxf + dyf * dyf;
            const Px t = load_px(sm, plane, rowo + kx);
            const float dA = dist3(c.a, t.a), dB = dist3(c.b, t.b);
            const float dAl = dist3(c.al, t.al), dN = dist3(c.n, t.n);
            const float eA = -b0 * dA - b2 * dAl - b3 * dN - b4 * pd;
            const float eB = -b1 * dB - b2 * dAl - b3 * dN - b4 * pd;
            const float wA = __expf(eA), wB = __expf(eB);
            const float kA[4] = {dA, dAl, dN, pd}, kB[4] = {dB, dAl, dN, pd};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float da = wA * (-kA[k]), db = wB * (-kB[k]);
                pA[k].x = fmaf(da, t.a[0], pA[k].x);
                pA[k].y = fmaf(da, t.a[1], pA[k].y);
                pA[k].z = fmaf(da, t.a[2], pA[k].z);
                pA[k].w += da;
                pB[k].x = fmaf(db, t.b[0], pB[k].x);
                pB[k].y = fmaf(db, t.b[1], pB[k].y);
                pB[k].z = fmaf(db, t.b[2], pB[k].z);
                pB[k].w += db;
            }
        }
    }
    float oA[4], oB[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        oA[k] = fmaf(gwA, pA[k].w, fmaf(gA.z, pA[k].z, fmaf(gA.x, pA[k].x, gA.y * pA[k].y)));
        oB[k] = fmaf(gwB, pB[k].w, fmaf(gB.z, pB[k].z, fmaf(gB.x, pB[k].x, gB.y * pB[k].y)));
    }
    float *o = gband + 5 * p;
    o[0] = oA[0];
    o[1] = oB[0];
    o[2] = oA[1] + oB[1];
    o[3] = oA[2] + oB[2];
    o[4] = oA[3] + oB[3];
}

}  // namespace

static cudaError_t sf_prepare(const void *fn, int hw, size_t *smem)
{
    *smem = sf_smem(hw);
    if (*smem > 220 * 1024 || 2 * hw + 1 > kMaxTable * 2) return cudaErrorInvalidConfiguration;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
}

cudaError_t launch_spatial_filter(const float *imga, const float *imgb, const float *albedo,
                                  const float *normal, const float *band, float *acca,
                                  float *accb, float *wsa, float *wsb, int B, int H, int W,
                                  int win, cudaStream_t st)
{
    const int hw = win / 2;
    size_t smem;
    cudaError_t e = sf_prepare((const void *)sf_forward_kernel, hw, &smem);
    if (e != cudaSuccess) return e;
    dim3 grid((W + kBX - 1) / kBX, (H + kBY - 1) / kBY, B);
    sf_forward_kernel<<<grid, dim3(kBX, kBY), smem, st>>>(imga, imgb, albedo, normal, band, acca,
                                                          accb, wsa, wsb, H, W, hw);
    return cudaGetLastError();
}

cudaError_t launch_spatial_filter_grad(const float *gacca, const float *gaccb, const float *gwsa,
                                       const float *gwsb, const float *imga, const float *imgb,
                                       const float *albedo, const float *normal,
                                       const float *band, float *gband, int B, int H, int W,
                                       int win, cudaStream_t st)
{
    const int hw = win / 2;
    size_t smem;
    cudaError_t e = sf_prepare((const void *)sf_grad_kernel, hw, &smem);
    if (e != cudaSuccess) return e;
    dim3 grid((W + kBX - 1) / kBX, (H + kBY - 1) / kBY, B);
    sf_grad_kernel<<<grid, dim3(kBX, kBY), smem, st>>>(gacca, gaccb, gwsa, gwsb, imga, imgb,
                                                       albedo, normal, band, gband, H, W, hw);
    return cudaGetLastError();
}

}  // namespace cd
