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

CD_DEV AggOut aggregate(const AggIn &in, float inv_n)
{
    AggOut r;
    const float d1 = in.w1 + 1e-4f, d2 = in.w2 + 1e-4f, d12 = (in.w1 + in.w2) + 1e-4f;
    const float op = in.opac > 0.f ? 1.f : 0.f;
    const float s = in.succ * in.succ_prev;
    const float a = s * in.alpha + (1.f - s);
    const float c = 0.25f * op * inv_n;
    float ga = 0.f, gw1 = 0.f, gw2 = 0.f, loss = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float o1s = in.s1[k] / d1, o2s = in.s2[k] / d2;
        const float oall = (in.s1[k] + in.s2[k]) / d12;
        const float pv = in.prev[k];
        const float ol = (a * oall + (1.f - a) * pv) * op;
        r.out_log[k] = ol;
        r.out[k] = fmaxf(0.f, expm1f(ol));
        const float o1 = a * o1s + (1.f - a) * pv, o2 = a * o2s + (1.f - a) * pv;
        const float n1 = in.l1[k] * in.l1[k] + 1e-2f, n2 = in.l2[k] * in.l2[k] + 1e-2f;
        const float p1 = in.pl1[k] * in.pl1[k] + 1e-2f, p2 = in.pl2[k] * in.pl2[k] + 1e-2f;
        const float e1 = o1 - in.l1[k], e2 = o2 - in.l2[k], f1 = o1 - in.pl1[k], f2 = o2 - in.pl2[k];
        const float spatial = (e1 * e1 / n1 + e2 * e2 / n2) * 0.5f;
        const float temporal = (f1 * f1 / p1 + f2 * f2 / p2) * 0.5f;
        r.loss_ch[k] = (spatial + temporal) * 0.5f * op;
        loss += r.loss_ch[k];
        const float go1 = c * (2.f * e1 / n1 + 2.f * f1 / p1);
        const float go2 = c * (2.f * e2 / n2 + 2.f * f2 / p2);
        r.g_s1[k] = go1 * a / d1;
        r.g_s2[k] = go2 * a / d2;
        gw1 += go1 * a * in.s1[k];
        gw2 += go2 * a * in.s2[k];
        ga += go1 * (o1s - pv) + go2 * (o2s - pv);
    }
    r.g_w1 = -gw1 / (d1 * d1);
    r.g_w2 = -gw2 / (d2 * d2);
    r.g_alpha = s * ga;
    r.loss = loss;
    return r;
}

// Block-wide sum of v written to partial[block]; partial sums are reduced
// in index order by loss_reduce_kernel, so the mean is deterministic.
CD_DEV void block_partial(float v, float *partial, int nthreads)
{
    __shared__ float red[32];
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid < 32) {
        float u = tid < (nthreads + 31) / 32 ? red[tid] : 0.f;
        for (int m = 16; m > 0; m >>= 1) u += __shfl_xor_sync(0xffffffffu, u, m);
        if (tid == 0) partial[(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = u;
    }
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

// ---------------------------------------------------------------------------
// Chosen path: spatial filter + aggregation loss + band gradient in one pass.
// The window sweep is the forward kernel's (same order, same arithmetic, so
// the filter sums equal cd_spatial_filter's bit for bit) extended with the
// band partials of the gradient kernel; the epilogue evaluates the loss and
// its gradient at the pixel and dots it with the partials.
// ---------------------------------------------------------------------------
constexpr int kBX = 32, kBY = 8, kPlanes = 12;

__global__ void __launch_bounds__(256) filter_aggregate_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb, const float *__restrict__ albedo,
    const float *__restrict__ normal, const float *__restrict__ band, AggPtrs P,
    float *__restrict__ gband, int H, int W, int hw, float inv_n)
{
    extern __shared__ float sm[];
    const int tw = kBX + 2 * hw, th = kBY + 2 * hw, plane = tw * th;
    float *tab = sm + kPlanes * plane;
    const size_t px = (size_t)H * W, b = blockIdx.z;
    const float *ia = imga + 3 * px * b, *ib = imgb + 3 * px * b;
    const float *al = albedo + 3 * px * b, *nr = normal + 3 * px * b;
    {
        const int x0 = blockIdx.x * kBX - hw, y0 = blockIdx.y * kBY - hw;
        const int tid = threadIdx.y * kBX + threadIdx.x;
        for (int t = tid; t < plane; t += kBX * kBY) {
            const int ty = t / tw, tx = t - ty * tw;
            const int gx = min(max(mirror(x0 + tx, W), 0), W - 1);
            const int gy = min(max(mirror(y0 + ty, H), 0), H - 1);
            const size_t q = (size_t)gy * W + gx;
            const float3 a = ld3(ia, q), c = ld3(ib, q), l = ld3(al, q), n = ld3(nr, q);
            const float v[12] = {a.x, a.y, a.z, c.x, c.y, c.z, l.x, l.y, l.z, n.x, n.y, n.z};
#pragma unroll
            for (int k = 0; k < 12; ++k) sm[k * plane + t] = v[k];
        }
        for (int k = tid; k <= 2 * hw; k += kBX * kBY) tab[k] = (float)(hw - k) / (float)hw;
    }
    __syncthreads();

    const int cx = blockIdx.x * kBX + threadIdx.x, cy = blockIdx.y * kBY + threadIdx.y;
    const bool ok = cx < W && cy < H;
    float loss = 0.f;
    if (ok) {
        const size_t p = b * px + (size_t)cy * W + cx;
        const float b0 = __ldg(band + 5 * p), b1 = __ldg(band + 5 * p + 1), b2 = __ldg(band + 5 * p + 2);
        const float b3 = __ldg(band + 5 * p + 3), b4 = __ldg(band + 5 * p + 4);
        const int co = (threadIdx.y + hw) * tw + threadIdx.x + hw;
        float c[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) c[k] = sm[k * plane + co];

        float aA[3] = {0.f, 0.f, 0.f}, aB[3] = {0.f, 0.f, 0.f}, sA = 0.f, sB = 0.f;
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
                const int o = rowo + kx;
                float t[12];
#pragma unroll
                for (int k = 0; k < 12; ++k) t[k] = sm[k * plane + o];
                const float dA = norm2(c[0] - t[0], c[1] - t[1], c[2] - t[2]);
                const float dB = norm2(c[3] - t[3], c[4] - t[4], c[5] - t[5]);
                const float dAl = norm2(c[6] - t[6], c[7] - t[7], c[8] - t[8]);
                const float dN = norm2(c[9] - t[9], c[10] - t[10], c[11] - t[11]);
                const float eA = -b0 * dA - b2 * dAl - b3 * dN - b4 * pd;
                const float eB = -b1 * dB - b2 * dAl - b3 * dN - b4 * pd;
                const float wA = __expf(eA), wB = __expf(eB);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    aA[k] = fmaf(wA, t[k], aA[k]);
                    aB[k] = fmaf(wB, t[3 + k], aB[k]);
                }
                sA += wA;
                sB += wB;
                const float kA[4] = {dA, dAl, dN, pd}, kB[4] = {dB, dAl, dN, pd};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float da = wA * (-kA[k]), db = wB * (-kB[k]);
                    pA[k].x = fmaf(da, t[0], pA[k].x);
                    pA[k].y = fmaf(da, t[1], pA[k].y);
                    pA[k].z = fmaf(da, t[2], pA[k].z);
                    pA[k].w += da;
                    pB[k].x = fmaf(db, t[3], pB[k].x);
                    pB[k].y = fmaf(db, t[4], pB[k].y);
                    pB[k].z = fmaf(db, t[5], pB[k].z);
                    pB[k].w += db;
                }
            }
        }
        AggIn in;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            in.s1[k] = aA[k];
            in.s2[k] = aB[k];
            in.prev[k] = __ldg(P.prev + 3 * p + k);
            in.l1[k] = c[3 + k];                       // label1 = ols2
            in.l2[k] = c[k];                           // label2 = ols1
            in.pl1[k] = __ldg(P.pl1 + 3 * p + k);      // prev_label1 = prev_ols2
            in.pl2[k] = __ldg(P.pl2 + 3 * p + k);      // prev_label2 = prev_ols1
        }
        in.w1 = sA;
        in.w2 = sB;
        in.alpha = __ldg(P.alpha + p);
        in.succ = __ldg(P.succ + p);
        in.succ_prev = __ldg(P.succ_prev + p);
        in.opac = __ldg(P.opac + p);
        const AggOut r = aggregate(in, inv_n);
        st3(P.out_log, p, make_float3(r.out_log[0], r.out_log[1], r.out_log[2]));
        st3(P.out, p, make_float3(r.out[0], r.out[1], r.out[2]));
        P.g_alpha[p] = r.g_alpha;
        loss = r.loss;
        float oA[4], oB[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            oA[k] = fmaf(r.g_w1, pA[k].w, fmaf(r.g_s1[2], pA[k].z, fmaf(r.g_s1[0], pA[k].x, r.g_s1[1] * pA[k].y)));
            oB[k] = fmaf(r.g_w2, pB[k].w, fmaf(r.g_s2[2], pB[k].z, fmaf(r.g_s2[0], pB[k].x, r.g_s2[1] * pB[k].y)));
        }
        float *o = gband + 5 * p;
        o[0] = oA[0];
        o[1] = oB[0];
        o[2] = oA[1] + oB[1];
        o[3] = oA[2] + oB[2];
        o[4] = oA[3] + oB[3];
    }
    block_partial(loss, P.partial, kBX * kBY);
}

}  // namespace

size_t aggregation_partials(int B, int H, int W) { return (size_t)((W + 31) / 32) * ((H + 7) / 8) * B; }

cudaError_t launch_log1p(const float *a, const float *b, float *ya, float *yb, size_t n, cudaStream_t st)
{
    log1p_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, ya, yb, n);
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

size_t filter_aggregate_smem(int win)
{
    const int hw = win / 2;
    return (size_t)kPlanes * (kBX + 2 * hw) * (kBY + 2 * hw) * sizeof(float) + 256 * sizeof(float);
}

cudaError_t launch_filter_aggregate(const float *imga, const float *imgb, const float *albedo,
                                    const float *normal, const float *band, const AggArgs &A, float *gband,
                                    float *partial, float *avg, int B, int H, int W, int win, cudaStream_t st)
{
    AggPtrs P{nullptr, nullptr, nullptr, nullptr, A.alpha, A.succ, A.succ_prev, A.prev, A.opac, nullptr,
              nullptr, A.pl1, A.pl2, A.out_log, A.out, nullptr, nullptr, nullptr, nullptr, nullptr,
              A.g_alpha, partial};
    const int hw = win / 2;
    const size_t smem = filter_aggregate_smem(win);
    cudaError_t e = cudaFuncSetAttribute(filter_aggregate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const float inv_n = 1.f / (3.f * (float)B * (float)H * (float)W);
    dim3 block(kBX, kBY), grid((W + kBX - 1) / kBX, (H + kBY - 1) / kBY, B);
    filter_aggregate_kernel<<<grid, block, smem, st>>>(imga, imgb, albedo, normal, band, P, gband, H, W, hw,
                                                       inv_n);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    loss_reduce_kernel<<<1, 1024, 0, st>>>(partial, (int)(grid.x * grid.y * grid.z), inv_n, avg);
    return cudaGetLastError();
}

}  // namespace cd
