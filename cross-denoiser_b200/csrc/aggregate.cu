// Aggregation loss of the online training step, forward and backward, and
// its fusion with the spatial filter.
//
// Reference semantics: aggregation_loss, scripts/main.py:214-248, with the
// labels crossed as train_step sets them (label1 = ols2, label2 = ols1,
// prev_label1 = prev_ols2, prev_label2 = prev_ols1, :283-286), and the
// gradient TensorFlow derives for it (:302):
//   o1 = a * sum1 / (sumw1 + 1e-4) + (1 - a) * prev_out,  o2 likewise,
//   a  = s * alpha + (1 - s),  s = success * success_prev,
//   out = (a * (sum1 + sum2) / (sumw1 + sumw2 + 1e-4) + (1 - a) * prev_out) * op,
//   loss = 0.25 * op * sum_{o in o1,o2} [(o - l)^2/(l^2 + 1e-2) + (o - pl)^2/(pl^2 + 1e-2)],
//   avg_loss = mean(loss) over B*H*W*3 elements, op = opacity > 0.
// dL/dsum, dL/dsumw and dL/dalpha are closed-form per pixel, so the fused
// kernel evaluates them right after the filter sums of the same pixel and
// dots them with the band partials accumulated in the same window pass: one
// pass gives the filtered frame, the loss and dL/dband.
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "filter_sweep.cuh"

namespace cd {
namespace {

struct AggIn {
    float s1[3], w1, s2[3], w2;   // filter sums of buffers A and B
    float alpha, succ, succ_prev, opac;
    float prev[3], l1[3], l2[3], pl1[3], pl2[3];
};

struct AggOut {
    float out_log[3], out[3], loss_ch[3], loss;   // loss: sum of the three channels
    float g_s1[3], g_w1, g_s2[3], g_w2, g_alpha;
};

// The 41 quotients of a pixel share 15 denominators: each denominator's
// reciprocal is taken once (__fdividef, about 2 ulp; every denominator is at
// least 1e-4) and the quotients become products.  The plain aggregation
// kernel and the fused filter kernel both evaluate this function, so their
// results stay identical to each other; against the eager FP32 formulas they
// differ by a few ulp.
CD_DEV AggOut aggregate(const AggIn &in, float inv_n)
{
    AggOut r;
    const float d1 = in.w1 + 1e-4f, d2 = in.w2 + 1e-4f, d12 = (in.w1 + in.w2) + 1e-4f;
    const float r1 = __fdividef(1.f, d1), r2 = __fdividef(1.f, d2), r12 = __fdividef(1.f, d12);
    const float op = in.opac > 0.f ? 1.f : 0.f;
    const float s = in.succ * in.succ_prev;
    const float a = s * in.alpha + (1.f - s);
    const float c = 0.25f * op * inv_n;
    const float ar1 = a * r1, ar2 = a * r2;
    float ga = 0.f, gw1 = 0.f, gw2 = 0.f, loss = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float o1s = in.s1[k] * r1, o2s = in.s2[k] * r2;
        const float oall = (in.s1[k] + in.s2[k]) * r12;
        const float pv = in.prev[k];
        const float ol = (a * oall + (1.f - a) * pv) * op;
        r.out_log[k] = ol;
        r.out[k] = fmaxf(0.f, expm1f(ol));
        const float o1 = a * o1s + (1.f - a) * pv, o2 = a * o2s + (1.f - a) * pv;
        const float rn1 = __fdividef(1.f, in.l1[k] * in.l1[k] + 1e-2f), rn2 = __fdividef(1.f, in.l2[k] * in.l2[k] + 1e-2f);
        const float rp1 = __fdividef(1.f, in.pl1[k] * in.pl1[k] + 1e-2f);
        const float rp2 = __fdividef(1.f, in.pl2[k] * in.pl2[k] + 1e-2f);
        const float e1 = o1 - in.l1[k], e2 = o2 - in.l2[k], f1 = o1 - in.pl1[k], f2 = o2 - in.pl2[k];
        const float e1n = e1 * rn1, e2n = e2 * rn2, f1p = f1 * rp1, f2p = f2 * rp2;
        const float spatial = (e1 * e1n + e2 * e2n) * 0.5f;
        const float temporal = (f1 * f1p + f2 * f2p) * 0.5f;
        r.loss_ch[k] = (spatial + temporal) * 0.5f * op;
        loss += r.loss_ch[k];
        const float go1 = c * (2.f * e1n + 2.f * f1p);
        const float go2 = c * (2.f * e2n + 2.f * f2p);
        r.g_s1[k] = go1 * ar1;
        r.g_s2[k] = go2 * ar2;
        gw1 += go1 * a * in.s1[k];
        gw2 += go2 * a * in.s2[k];
        ga += go1 * (o1s - pv) + go2 * (o2s - pv);
    }
    r.g_w1 = -gw1 * (r1 * r1);
    r.g_w2 = -gw2 * (r2 * r2);
    r.g_alpha = s * ga;
    r.loss = loss;
    return r;
}

// Block-wide sum of v written to partial[block]; partial sums are reduced
// in index order by loss_reduce_kernel, so the mean is deterministic.
// block_partial_at writes it to partial[index] and ends with a barrier, so
// a persistent CTA can call it once per tile.
CD_DEV void block_partial_at(float v, float *partial, int index, int nthreads)
{
    __shared__ float red[32];
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid < 32) {
        float u = tid < (nthreads + 31) / 32 ? red[tid] : 0.f;
        for (int m = 16; m > 0; m >>= 1) u += __shfl_xor_sync(0xffffffffu, u, m);
        if (tid == 0) partial[index] = u;
    }
    __syncthreads();
}

CD_DEV void block_partial(float v, float *partial, int nthreads)
{
    block_partial_at(v, partial, (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x, nthreads);
}

__global__ void __launch_bounds__(1024) loss_reduce_kernel(const float *__restrict__ partial, int n,
                                                           float inv_n, float *__restrict__ avg)
{
    __shared__ float red[32];
    float v = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        float u = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
        for (int m = 16; m > 0; m >>= 1) u += __shfl_xor_sync(0xffffffffu, u, m);
        if (threadIdx.x == 0) *avg = u * inv_n;
    }
}

__global__ void __launch_bounds__(256) log1p_kernel(const float *__restrict__ a, const float *__restrict__ b,
                                                    float *__restrict__ ya, float *__restrict__ yb, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        ya[i] = log1pf(__ldg(a + i));
        yb[i] = log1pf(__ldg(b + i));
    }
}

// 16-byte aligned buffers: each thread takes kLogVec float4 of both inputs,
// all loads issued before the first log1pf, so that enough bytes are in
// flight to cover the DRAM latency.
constexpr int kLogVec = 2;
__global__ void __launch_bounds__(256) log1p4_kernel(const float4 *__restrict__ a, const float4 *__restrict__ b,
                                                     float4 *__restrict__ ya, float4 *__restrict__ yb, size_t n4)
{
    const size_t i0 = ((size_t)blockIdx.x * kLogVec) * blockDim.x + threadIdx.x;
    float4 va[kLogVec], vb[kLogVec];
#pragma unroll
    for (int k = 0; k < kLogVec; ++k) {
        const size_t i = i0 + (size_t)k * blockDim.x;
        if (i < n4) {
            va[k] = __ldg(a + i);
            vb[k] = __ldg(b + i);
        }
    }
#pragma unroll
    for (int k = 0; k < kLogVec; ++k) {
        const size_t i = i0 + (size_t)k * blockDim.x;
        if (i < n4) {
            ya[i] = make_float4(log1pf(va[k].x), log1pf(va[k].y), log1pf(va[k].z), log1pf(va[k].w));
            yb[i] = make_float4(log1pf(vb[k].x), log1pf(vb[k].y), log1pf(vb[k].z), log1pf(vb[k].w));
        }
    }
}

struct AggPtrs {
    const float *s1, *w1, *s2, *w2, *alpha, *succ, *succ_prev, *prev, *opac, *l1, *l2, *pl1, *pl2;
    float *out_log, *out, *loss, *g_s1, *g_w1, *g_s2, *g_w2, *g_alpha, *partial;
};

// ---------------------------------------------------------------------------
// Plain path: the aggregation loss forward + backward, one thread per pixel.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) aggregation_kernel(AggPtrs P, int H, int W, float inv_n)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const bool ok = x < W && y < H;
    float loss = 0.f;
    if (ok) {
        const size_t p = ((size_t)blockIdx.z * H + y) * W + x;
        AggIn in;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            in.s1[k] = __ldg(P.s1 + 3 * p + k);
            in.s2[k] = __ldg(P.s2 + 3 * p + k);
            in.prev[k] = __ldg(P.prev + 3 * p + k);
            in.l1[k] = __ldg(P.l1 + 3 * p + k);
            in.l2[k] = __ldg(P.l2 + 3 * p + k);
            in.pl1[k] = __ldg(P.pl1 + 3 * p + k);
            in.pl2[k] = __ldg(P.pl2 + 3 * p + k);
        }
        in.w1 = __ldg(P.w1 + p);
        in.w2 = __ldg(P.w2 + p);
        in.alpha = __ldg(P.alpha + p);
        in.succ = __ldg(P.succ + p);
        in.succ_prev = __ldg(P.succ_prev + p);
        in.opac = __ldg(P.opac + p);
        const AggOut r = aggregate(in, inv_n);
        st3(P.out_log, p, make_float3(r.out_log[0], r.out_log[1], r.out_log[2]));
        st3(P.out, p, make_float3(r.out[0], r.out[1], r.out[2]));
        st3(P.g_s1, p, make_float3(r.g_s1[0], r.g_s1[1], r.g_s1[2]));
        st3(P.g_s2, p, make_float3(r.g_s2[0], r.g_s2[1], r.g_s2[2]));
        P.g_w1[p] = r.g_w1;
        P.g_w2[p] = r.g_w2;
        P.g_alpha[p] = r.g_alpha;
        if (P.loss) st3(P.loss, p, make_float3(r.loss_ch[0], r.loss_ch[1], r.loss_ch[2]));
        loss = r.loss;
    }
    block_partial(loss, P.partial, blockDim.x * blockDim.y);
}

// Epilogue of the fused filter kernels at pixel p: the aggregation loss and
// its gradient from the window sums, written outputs, dL/dband from the
// partials; returns the pixel's loss (sum over its three channels).
CD_DEV float filter_epilogue(const fsw::Sums &s, const fsw::Centre &c, const AggPtrs &P, size_t p,
                             float *__restrict__ gband, float inv_n)
{
    AggIn in;
    in.s1[0] = fsw::lo(s.acc_x);
    in.s1[1] = fsw::lo(s.acc_y);
    in.s1[2] = fsw::lo(s.acc_z);
    in.s2[0] = fsw::hi(s.acc_x);
    in.s2[1] = fsw::hi(s.acc_y);
    in.s2[2] = fsw::hi(s.acc_z);
    in.w1 = fsw::lo(s.acc_w);
    in.w2 = fsw::hi(s.acc_w);
    // labels crossed as train_step sets them: label1 = ols2, label2 = ols1
    in.l1[0] = fsw::hi(c.ab_x);
    in.l1[1] = fsw::hi(c.ab_y);
    in.l1[2] = fsw::hi(c.ab_z);
    in.l2[0] = fsw::lo(c.ab_x);
    in.l2[1] = fsw::lo(c.ab_y);
    in.l2[2] = fsw::lo(c.ab_z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        in.prev[k] = __ldg(P.prev + 3 * p + k);
        in.pl1[k] = __ldg(P.pl1 + 3 * p + k);      // prev_label1 = prev_ols2
        in.pl2[k] = __ldg(P.pl2 + 3 * p + k);      // prev_label2 = prev_ols1
    }
    in.alpha = __ldg(P.alpha + p);
    in.succ = __ldg(P.succ + p);
    in.succ_prev = __ldg(P.succ_prev + p);
    in.opac = __ldg(P.opac + p);
    const AggOut r = aggregate(in, inv_n);
    st3(P.out_log, p, make_float3(r.out_log[0], r.out_log[1], r.out_log[2]));
    st3(P.out, p, make_float3(r.out[0], r.out[1], r.out[2]));
    P.g_alpha[p] = r.g_alpha;
    fsw::band_grad(s, make_float3(r.g_s1[0], r.g_s1[1], r.g_s1[2]), make_float3(r.g_s2[0], r.g_s2[1], r.g_s2[2]),
                   r.g_w1, r.g_w2, gband + 5 * p);
    return r.loss;
}

// ---------------------------------------------------------------------------
// Chosen path: spatial filter + aggregation loss + band gradient in one pass.
// The window sweep is the forward kernel's (same order, same arithmetic)
// extended with the band partials of the gradient kernel; the epilogue
// evaluates the loss and its gradient at the pixel and dots it with the
// partials.  Its weights are exp(e) = 2^(e log2 e) on ex2.approx.ftz
// (fsw::kExp2Ftz): the same values as the plain kernels' __expf wherever the
// weight is a normal float, zero where it would be subnormal (below 2^-126),
// so its sums equal cd_spatial_filter's except for contributions below the
// smallest normal float.  Launch bound 2 CTAs per SM: 120 registers without
// spills (a bound of 3 allows 80 and spills in the sweep); measured 736
// against 745 us at 1920x1080, window 11.
// ---------------------------------------------------------------------------
template <int HW>
__global__ void __launch_bounds__(256, 2) filter_aggregate_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb, const float *__restrict__ albedo,
    const float *__restrict__ normal, const float *__restrict__ band, AggPtrs P,
    float *__restrict__ gband, int H, int W, int hw_rt, float inv_n)
{
    extern __shared__ ulonglong2 tile[];
    const int hw = HW > 0 ? HW : hw_rt;
    const int tw = fsw::kBX + 2 * hw, th = fsw::kBY + 2 * hw;
    fsw::f2 *pdtab = reinterpret_cast<fsw::f2 *>(tile + 3 * tw * th);
    const size_t px = (size_t)H * W, b = blockIdx.z;
    fsw::stage(tile, pdtab, imga + 3 * px * b, imgb + 3 * px * b, albedo + 3 * px * b, normal + 3 * px * b,
               H, W, hw);
    __syncthreads();

    const int cx = blockIdx.x * fsw::kBX + threadIdx.x, cy = blockIdx.y * fsw::kBY + threadIdx.y;
    float loss = 0.f;
    if (cx < W && cy < H) {
        const size_t p = b * px + (size_t)cy * W + cx;
        const fsw::Centre c = fsw::centre(tile, hw, band + 5 * p);
        fsw::Sums s;
        fsw::zero(s);
        fsw::sweep<HW, true, true, fsw::kExp2Ftz>(tile, pdtab, hw, c, s);
        loss = filter_epilogue(s, c, P, p, gband, inv_n);
    }
    block_partial(loss, P.partial, fsw::kBX * fsw::kBY);
}


}  // namespace

size_t aggregation_partials(int B, int H, int W) { return (size_t)((W + 31) / 32) * ((H + 7) / 8) * B; }

cudaError_t launch_log1p(const float *a, const float *b, float *ya, float *yb, size_t n, cudaStream_t st)
{
    const bool vec = n % 4 == 0 && ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
                                     reinterpret_cast<uintptr_t>(ya) | reinterpret_cast<uintptr_t>(yb)) & 15) == 0;
    if (vec) {
        const size_t n4 = n / 4, per = (size_t)256 * kLogVec;
        log1p4_kernel<<<(unsigned)((n4 + per - 1) / per), 256, 0, st>>>(
            reinterpret_cast<const float4 *>(a), reinterpret_cast<const float4 *>(b), reinterpret_cast<float4 *>(ya),
            reinterpret_cast<float4 *>(yb), n4);
    } else {
        log1p_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, ya, yb, n);
    }
    return cudaGetLastError();
}

cudaError_t launch_aggregation(const AggArgs &A, float *partial, float *avg, int B, int H, int W,
                               cudaStream_t st)
{
    AggPtrs P{A.s1, A.w1, A.s2, A.w2, A.alpha, A.succ, A.succ_prev, A.prev, A.opac, A.l1, A.l2, A.pl1, A.pl2,
              A.out_log, A.out, A.loss, A.g_s1, A.g_w1, A.g_s2, A.g_w2, A.g_alpha, partial};
    const float inv_n = 1.f / (3.f * (float)B * (float)H * (float)W);
    dim3 block(32, 8), grid((W + 31) / 32, (H + 7) / 8, B);
    aggregation_kernel<<<grid, block, 0, st>>>(P, H, W, inv_n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    loss_reduce_kernel<<<1, 1024, 0, st>>>(partial, (int)(grid.x * grid.y * grid.z), inv_n, avg);
    return cudaGetLastError();
}

size_t filter_aggregate_smem(int win) { return fsw::smem_bytes(win / 2); }

cudaError_t launch_filter_aggregate(const float *imga, const float *imgb, const float *albedo,
                                    const float *normal, const float *band, const AggArgs &A, float *gband,
                                    float *partial, float *avg, int B, int H, int W, int win, cudaStream_t st)
{
    AggPtrs P{nullptr, nullptr, nullptr, nullptr, A.alpha, A.succ, A.succ_prev, A.prev, A.opac, nullptr,
              nullptr, A.pl1, A.pl2, A.out_log, A.out, nullptr, nullptr, nullptr, nullptr, nullptr,
              A.g_alpha, partial};
    const int hw = win / 2;
    const size_t smem = fsw::smem_bytes(hw);
    const float inv_n = 1.f / (3.f * (float)B * (float)H * (float)W);
    dim3 block(fsw::kBX, fsw::kBY), grid((W + fsw::kBX - 1) / fsw::kBX, (H + fsw::kBY - 1) / fsw::kBY, B);
    auto go = [&](auto kern) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, block, smem, st>>>(imga, imgb, albedo, normal, band, P, gband, H, W, hw, inv_n);
        return cudaGetLastError();
    };
    cudaError_t e;
    switch (hw) {
    case 3: e = go(filter_aggregate_kernel<3>); break;
    case 5: e = go(filter_aggregate_kernel<5>); break;
    case 7: e = go(filter_aggregate_kernel<7>); break;
    default: e = go(filter_aggregate_kernel<0>); break;
    }
    if (e != cudaSuccess) return e;
    loss_reduce_kernel<<<1, 1024, 0, st>>>(partial, (int)(grid.x * grid.y * grid.z), inv_n, avg);
    return cudaGetLastError();
}

}  // namespace cd
