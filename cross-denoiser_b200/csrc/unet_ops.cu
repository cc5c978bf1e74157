// The U-Net's non-convolution layers, their backward passes, the gradient
// reductions and the optimizer (scripts/main.py:74-118, 300-303):
//   input packing      Concatenate of the five 3-channel inputs (:101-102)
//   Conv2DTranspose    kernel 1, stride 2, 'same' (:92, :96): out[2i,2j] =
//                      K x[i,j] + b, every other position b; Keras kernel
//                      layout [1][1][cout][cin]
//   head               Conv2D(6, 1) in fp32, band = 1 / (p^2 + 1e-4),
//                      alpha = sigmoid (:106-111)
//   max-pool backward  the gradient goes to the first maximum of each 2x2
//                      window (row-major), added to the skip connection's
//                      gradient, times the ReLU derivative
//   Adam               Keras semantics: m += (g - m)(1 - b1),
//                      v += (g^2 - v)(1 - b2),
//                      w -= lr sqrt(1 - b2^t) / (1 - b1^t) m / (sqrt(v) + eps)
// Per-block partial sums of the parameter gradients are reduced in a fixed
// order by reduce_kernel, so the gradients are deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "unet.cuh"
#include "unet_ops.cuh"

namespace cd {
namespace unet {
namespace {

CD_DEV void ld8(const __nv_bfloat16 *p, float *v)
{
    const uint4 raw = *reinterpret_cast<const uint4 *>(p);
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&raw);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float2 f = __bfloat1622float2(h[e]);
        v[2 * e] = f.x;
        v[2 * e + 1] = f.y;
    }
}
CD_DEV void st8(__nv_bfloat16 *p, const float *v)
{
    uint4 o;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
    for (int e = 0; e < 4; ++e) h[e] = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
    *reinterpret_cast<uint4 *>(p) = o;
}

// [ols1, ols2, prev_out, albedo, normal] (fp32, 3 channels each) -> bf16, 16
// channels (15 + zero) in two row-chunk planes; n = B * H * W pixels, W wide
__global__ void __launch_bounds__(256) pack_input_kernel(const float *__restrict__ a, const float *__restrict__ b,
                                                         const float *__restrict__ c, const float *__restrict__ d,
                                                         const float *__restrict__ e, __nv_bfloat16 *__restrict__ x,
                                                         size_t n, int W)
{
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int row = (int)(p / W), px = (int)(p - (size_t)row * W);
    float v[16];
    const float *src[5] = {a, b, c, d, e};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        v[3 * k] = __ldg(src[k] + 3 * p);
        v[3 * k + 1] = __ldg(src[k] + 3 * p + 1);
        v[3 * k + 2] = __ldg(src[k] + 3 * p + 2);
    }
    v[15] = 0.f;
    st8(x + act_idx(0, row, 0, px, 0, W, 2) * 8, v);
    st8(x + act_idx(0, row, 1, px, 0, W, 2) * 8, v + 8);
}

// Conv2DTranspose(kernel 1, stride 2) forward, one thread per input pixel
// (i, j): output (2i, 2j) = K x + b (each channel summed over ci in order,
// K rows read as float4), outputs (2i, 2j + 1), (2i + 1, 2j), (2i + 1, 2j + 1)
// = b.
template <int CI, int CO>
__global__ void __launch_bounds__(256) tconv_fwd_kernel(const __nv_bfloat16 *__restrict__ in,
                                                        const float *__restrict__ K, const float *__restrict__ bias,
                                                        __nv_bfloat16 *__restrict__ out, int Hi, int Wi, int B)
{
    __shared__ __align__(16) float sK[CO * CI + CO];
    for (int i = threadIdx.x; i < CO * CI + CO; i += blockDim.x) sK[i] = i < CO * CI ? K[i] : bias[i - CO * CI];
    __syncthreads();
    const int Ho = 2 * Hi, Wo = 2 * Wi;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)B * Hi * Wi) return;
    const int xi = (int)(p % Wi), yi = (int)((p / Wi) % Hi), b = (int)(p / ((size_t)Wi * Hi));
    float x[CI];
#pragma unroll
    for (int c = 0; c < CI; c += 8) ld8(in + act_idx(b, yi, c / 8, xi, Hi, Wi, CI / 8) * 8, x + c);
    float o[CO], ob[CO];
#pragma unroll
    for (int co = 0; co < CO; ++co) {
        ob[co] = sK[CO * CI + co];
        float s = ob[co];
        const float4 *kr = reinterpret_cast<const float4 *>(sK + co * CI);
#pragma unroll
        for (int c4 = 0; c4 < CI / 4; ++c4) {
            const float4 k4 = kr[c4];
            s = fmaf(k4.x, x[4 * c4], s);
            s = fmaf(k4.y, x[4 * c4 + 1], s);
            s = fmaf(k4.z, x[4 * c4 + 2], s);
            s = fmaf(k4.w, x[4 * c4 + 3], s);
        }
        o[co] = s;
    }
#pragma unroll
    for (int c = 0; c < CO; c += 8) {
        st8(out + act_idx(b, 2 * yi, c / 8, 2 * xi, Ho, Wo, CO / 8) * 8, o + c);
        st8(out + act_idx(b, 2 * yi, c / 8, 2 * xi + 1, Ho, Wo, CO / 8) * 8, ob + c);
        st8(out + act_idx(b, 2 * yi + 1, c / 8, 2 * xi, Ho, Wo, CO / 8) * 8, ob + c);
        st8(out + act_idx(b, 2 * yi + 1, c / 8, 2 * xi + 1, Ho, Wo, CO / 8) * 8, ob + c);
    }
}

// Conv2DTranspose backward: for every chunk of kN input pixels, d_in =
// K^T d_out[2i,2j] (times the ReLU derivative of `in`) and the chunk's
// contribution to dK[co][ci] and db[co] (db over all four output positions
// of each input pixel).  Blocks walk chunks blockIdx.x, + gridDim.x, ...
// and keep their dK / db sums in registers: one partial row per block.
template <int CI, int CO, int kN>
__global__ void __launch_bounds__(kN) tconv_bwd_kernel(const __nv_bfloat16 *__restrict__ in,
                                                        const __nv_bfloat16 *__restrict__ dout,
                                                        const float *__restrict__ K,
                                                        __nv_bfloat16 *__restrict__ dz_in, float *__restrict__ partial,
                                                        int Hi, int Wi, int B)
{
    // dK in 4 x 4 register tiles: kTiles tiles cover CO x CI, and the
    // threads split into kGroups pixel groups, each summing its share of a
    // chunk's pixels (in order) into every tile; the groups' sums are added
    // in group order at the end.  Then db.
    constexpr int TM = 4, TN = 4, kTiles = (CO / TM) * (CI / TN), kGroups = kN / kTiles;
    static_assert(kGroups >= 1 && kGroups * kTiles == kN && kN % kGroups == 0, "tiles x groups cover the block");
    __shared__ __align__(16) float sK[CO * CI];
    __shared__ float sx[kN][CI + 1], sd[kN][CO + 1], sb[kN][CO + 1];
    for (int i = threadIdx.x; i < CO * CI; i += blockDim.x) sK[i] = K[i];
    const size_t n = (size_t)B * Hi * Wi, nchunk = (n + kN - 1) / kN;
    const int t = threadIdx.x;
    const int tile = t % kTiles, grp = t / kTiles;
    const int tci = tile % (CI / TN), tco = tile / (CI / TN);
    const int ci0 = TN * tci, co0 = TM * tco;
    constexpr int kPer = kN / kGroups;   // pixels of a chunk per group
    float acc[TM][TN];
#pragma unroll
    for (int a = 0; a < TM; ++a)
#pragma unroll
        for (int c = 0; c < TN; ++c) acc[a][c] = 0.f;
    float bacc = 0.f;
    for (size_t chunk = blockIdx.x; chunk < nchunk; chunk += gridDim.x) {
        const size_t p = chunk * kN + t;
        float x[CI], d[CO];
#pragma unroll
        for (int c = 0; c < CI; ++c) x[c] = 0.f;
#pragma unroll
        for (int c = 0; c < CO; ++c) d[c] = 0.f;
        float bsum[CO];
#pragma unroll
        for (int c = 0; c < CO; ++c) bsum[c] = 0.f;
        const int xi = (int)(p % Wi), yi = (int)((p / Wi) % Hi), b = (int)(p / ((size_t)Wi * Hi));
        if (p < n) {
#pragma unroll
            for (int c = 0; c < CI; c += 8) ld8(in + act_idx(b, yi, c / 8, xi, Hi, Wi, CI / 8) * 8, x + c);
            const int Wo = 2 * Wi, Ho = 2 * Hi;
            for (int a = 0; a < 4; ++a) {
                const int yo = 2 * yi + (a >> 1), xo = 2 * xi + (a & 1);
                float g[CO];
#pragma unroll
                for (int c = 0; c < CO; c += 8) ld8(dout + act_idx(b, yo, c / 8, xo, Ho, Wo, CO / 8) * 8, g + c);
#pragma unroll
                for (int c = 0; c < CO; ++c) {
                    bsum[c] += g[c];
                    if (a == 0) d[c] = g[c];
                }
            }
        }
#pragma unroll
        for (int c = 0; c < CI; ++c) sx[t][c] = x[c];
#pragma unroll
        for (int c = 0; c < CO; ++c) {
            sd[t][c] = d[c];
            sb[t][c] = bsum[c];
        }
        __syncthreads();
        if (p < n) {
            // co outer, ci inner: each g[ci] still sums over co in order, and a
            // row of K is read as float4s
            float g[CI];
#pragma unroll
            for (int ci = 0; ci < CI; ++ci) g[ci] = 0.f;
#pragma unroll
            for (int co = 0; co < CO; ++co) {
                const float4 *kr = reinterpret_cast<const float4 *>(sK + co * CI);
#pragma unroll
                for (int c4 = 0; c4 < CI / 4; ++c4) {
                    const float4 k4 = kr[c4];
                    g[4 * c4] = fmaf(k4.x, d[co], g[4 * c4]);
                    g[4 * c4 + 1] = fmaf(k4.y, d[co], g[4 * c4 + 1]);
                    g[4 * c4 + 2] = fmaf(k4.z, d[co], g[4 * c4 + 2]);
                    g[4 * c4 + 3] = fmaf(k4.w, d[co], g[4 * c4 + 3]);
                }
            }
#pragma unroll
            for (int ci = 0; ci < CI; ++ci) g[ci] = x[ci] > 0.f ? g[ci] : 0.f;
#pragma unroll
            for (int c = 0; c < CI; c += 8) st8(dz_in + act_idx(b, yi, c / 8, xi, Hi, Wi, CI / 8) * 8, g + c);
        }
        for (int k = grp * kPer; k < (grp + 1) * kPer; ++k) {
            float dv[TM], xv[TN];
#pragma unroll
            for (int a = 0; a < TM; ++a) dv[a] = sd[k][co0 + a];
#pragma unroll
            for (int c = 0; c < TN; ++c) xv[c] = sx[k][ci0 + c];
#pragma unroll
            for (int a = 0; a < TM; ++a)
#pragma unroll
                for (int c = 0; c < TN; ++c) acc[a][c] = fmaf(dv[a], xv[c], acc[a][c]);
        }
        if (t < CO)
            for (int k = 0; k < kN; ++k) bacc += sb[k][t];
        __syncthreads();   // the chunk's tiles are read before the next one is written
    }
    float *out = partial + (size_t)blockIdx.x * (CO * CI + CO);
    if (kGroups == 1) {
#pragma unroll
        for (int a = 0; a < TM; ++a)
#pragma unroll
            for (int c = 0; c < TN; ++c) out[(co0 + a) * CI + ci0 + c] = acc[a][c];
    } else {
        // the groups' tiles through shared memory (sx is free now: kN x (CI + 1)
        // floats hold the kGroups x CO x CI sums)
        float *red = &sx[0][0];
        static_assert(kGroups * CO * CI <= kN * (CI + 1), "the group sums fit sx");
#pragma unroll
        for (int a = 0; a < TM; ++a)
#pragma unroll
            for (int c = 0; c < TN; ++c) red[(grp * CO + co0 + a) * CI + ci0 + c] = acc[a][c];
        __syncthreads();
        for (int j = t; j < CO * CI; j += kN) {
            float v = 0.f;
            for (int g = 0; g < kGroups; ++g) v += red[g * CO * CI + j];
            out[j] = v;
        }
    }
    if (t < CO) out[CO * CI + t] = bacc;
}

// Head: param = Kh^T c5_1 + bh (Kh[ci][co], 8 x 6), band = 1 / (p^2 + 1e-4), alpha = sigmoid(p5).
// A block's band values (five per pixel) go out through shared memory as
// float4 stores.
__global__ void __launch_bounds__(256) head_fwd_kernel(const __nv_bfloat16 *__restrict__ x, const float *__restrict__ K,
                                                       const float *__restrict__ bias, float *__restrict__ band,
                                                       float *__restrict__ alpha, size_t n)
{
    __shared__ float sK[54];
    __shared__ __align__(16) float sb[256 * 5];   // the block's band values, written out as float4
    const int tid = threadIdx.x;
    if (tid < 54) sK[tid] = tid < 48 ? K[tid] : bias[tid - 48];
    __syncthreads();
    const size_t p0 = (size_t)blockIdx.x * 256, p = p0 + tid;
    if (p < n) {
        float v[8];
        ld8(x + 8 * p, v);
        float q[6];
#pragma unroll
        for (int co = 0; co < 6; ++co) {
            float s = sK[48 + co];
#pragma unroll
            for (int ci = 0; ci < 8; ++ci) s = fmaf(sK[ci * 6 + co], v[ci], s);
            q[co] = s;
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) sb[5 * tid + k] = 1.f / (q[k] * q[k] + 1e-4f);
        alpha[p] = 1.f / (1.f + expf(-q[5]));
    }
    __syncthreads();
    const int cnt = 5 * (int)(n - p0 < 256 ? n - p0 : 256);
    float *dst = band + 5 * p0;
    int i = tid;
    if (!(reinterpret_cast<uintptr_t>(dst) & 15)) {
        for (; i < cnt / 4; i += 256) reinterpret_cast<float4 *>(dst)[i] = reinterpret_cast<const float4 *>(sb)[i];
        i = (cnt / 4) * 4 + tid;
    }
    for (; i < cnt; i += 256) dst[i] = sb[i];
}

// Head backward: dZ of c5_1 (times its ReLU derivative) and the block's
// partial sums of dKh[ci][co] and dbh[co].  Each thread walks pixels
// p = thread, thread + grid size, ... accumulating its 54 parameter-gradient
// terms in registers; the block then reduces them (lanes, then warps, in a
// fixed order) to one partial row.
constexpr int kHeadThreads = 256;
constexpr int kHeadMaxBlocks = 592;

__global__ void __launch_bounds__(kHeadThreads) head_bwd_kernel(const __nv_bfloat16 *__restrict__ x,
                                                                const float *__restrict__ K,
                                                                const float *__restrict__ bias,
                                                                const float *__restrict__ gband,
                                                                const float *__restrict__ galpha,
                                                                __nv_bfloat16 *__restrict__ dz,
                                                                float *__restrict__ partial, size_t n)
{
    __shared__ float sK[54];
    __shared__ float red[kHeadThreads / 32][54];
    const int tid = threadIdx.x;
    if (tid < 54) sK[tid] = tid < 48 ? K[tid] : bias[tid - 48];
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5;
    float acc[54];
#pragma unroll
    for (int j = 0; j < 54; ++j) acc[j] = 0.f;
    for (size_t p = (size_t)blockIdx.x * kHeadThreads + tid; p < n; p += (size_t)gridDim.x * kHeadThreads) {
        float v[8], g[6];
        ld8(x + 8 * p, v);
#pragma unroll
        for (int co = 0; co < 6; ++co) {
            float s = sK[48 + co];
#pragma unroll
            for (int ci = 0; ci < 8; ++ci) s = fmaf(sK[ci * 6 + co], v[ci], s);
            if (co < 5) {
                // d band / d s = -2 s / (s^2 + 1e-4)^2, with one fast
                // reciprocal (a gradient: FP32 tolerance, not the forward's
                // rounding)
                const float r = __fdividef(1.f, s * s + 1e-4f);
                g[co] = __ldg(gband + 5 * p + co) * (-2.f * s * r * r);
            } else {
                const float a = 1.f / (1.f + expf(-s));
                g[co] = __ldg(galpha + p) * a * (1.f - a);
            }
        }
        float d[8];
#pragma unroll
        for (int ci = 0; ci < 8; ++ci) {
            float s = 0.f;
#pragma unroll
            for (int co = 0; co < 6; ++co) s = fmaf(sK[ci * 6 + co], g[co], s);
            d[ci] = v[ci] > 0.f ? s : 0.f;
        }
        st8(dz + 8 * p, d);
#pragma unroll
        for (int ci = 0; ci < 8; ++ci)
#pragma unroll
            for (int co = 0; co < 6; ++co) acc[ci * 6 + co] = fmaf(v[ci], g[co], acc[ci * 6 + co]);
#pragma unroll
        for (int co = 0; co < 6; ++co) acc[48 + co] += g[co];
    }
#pragma unroll
    for (int j = 0; j < 54; ++j) {
        float s = acc[j];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp][j] = s;
    }
    __syncthreads();
    if (tid < 54) {
        float s = 0.f;
        for (int w = 0; w < kHeadThreads / 32; ++w) s += red[w][tid];
        partial[(size_t)blockIdx.x * 54 + tid] = s;
    }
}

// dZ = (maxpool backward of dpool + dskip) * [act > 0], C channels (multiple
// of 8).  One thread per pooled pixel (H and W even): it reads the four
// pixels of its 2x2 window once per 8-channel chunk; the pooled gradient
// goes to the first maximum of the window (row-major), as in the forward.
template <int C>
__global__ void __launch_bounds__(256) pool_bwd_kernel(const __nv_bfloat16 *__restrict__ act,
                                                       const __nv_bfloat16 *__restrict__ pooled,
                                                       const __nv_bfloat16 *__restrict__ dpool,
                                                       const __nv_bfloat16 *__restrict__ dskip,
                                                       __nv_bfloat16 *__restrict__ dz, int H, int W, int B)
{
    constexpr int NC = C / 8;
    const int PH = H / 2, PW = W / 2;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)B * PH * PW) return;
    const int px = (int)(q % PW), py = (int)((q / PW) % PH), b = (int)(q / ((size_t)PW * PH));
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        float m[8], dp[8], a[4][8], g[4][8];
        ld8(pooled + act_idx(b, py, c, px, PH, PW, NC) * 8, m);
        ld8(dpool + act_idx(b, py, c, px, PH, PW, NC) * 8, dp);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const size_t r = act_idx(b, 2 * py + (k >> 1), c, 2 * px + (k & 1), H, W, NC) * 8;
            ld8(act + r, a[k]);
            ld8(dskip + r, g[k]);
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            bool taken = false;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (!taken && a[k][e] == m[e]) {
                    g[k][e] += dp[e];
                    taken = true;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
#pragma unroll
            for (int e = 0; e < 8; ++e)
                if (!(a[k][e] > 0.f)) g[k][e] = 0.f;
            st8(dz + act_idx(b, 2 * py + (k >> 1), c, 2 * px + (k & 1), H, W, NC) * 8, g[k]);
        }
    }
}

// Fixed-order reduction of per-tile partial sums, one launch: a block owns
// 32 output columns (lane = column) and its 32 warps take the rows
// t = warp, warp + 32, ... in order; the warps' sums are then added in warp
// order.  The same partials always give the same result.
constexpr int kReduceWarps = 32;

__global__ void __launch_bounds__(32 * kReduceWarps) reduce_kernel(const float *__restrict__ partial,
                                                                   float *__restrict__ out, int n, int tiles)
{
    __shared__ float red[kReduceWarps][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = blockIdx.x * 32 + lane;
    float s = 0.f;
    if (j < n)
        for (int t = warp; t < tiles; t += kReduceWarps) s += __ldg(partial + (size_t)t * n + j);
    red[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && j < n) {
        float v = 0.f;
        for (int w = 0; w < kReduceWarps; ++w) v += red[w][lane];
        out[j] = v;
    }
}

// The update count lives in device memory (so a captured graph replays
// correct steps): t = *step + 1, lr_t = lr sqrt(1 - b2^t) / (1 - b1^t) in
// float as Keras computes it; step_kernel then advances the counter.
__global__ void __launch_bounds__(256) adam_kernel(float *__restrict__ w, const float *__restrict__ g,
                                                   float *__restrict__ m, float *__restrict__ v, int n,
                                                   const int *__restrict__ step, float lr, float b1, float b2,
                                                   float eps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float t = (float)(*step + 1);
    const float lr_t = lr * sqrtf(1.f - powf(b2, t)) / (1.f - powf(b1, t));
    const float gi = g[i];
    const float mi = m[i] + (gi - m[i]) * (1.f - b1);
    const float vi = v[i] + (gi * gi - v[i]) * (1.f - b2);
    m[i] = mi;
    v[i] = vi;
    w[i] -= (mi * lr_t) / (sqrtf(vi) + eps);
}

__global__ void step_kernel(int *step) { *step += 1; }

}  // namespace

cudaError_t launch_pack_input(const float *a, const float *b, const float *c, const float *d, const float *e,
                              __nv_bfloat16 *x, size_t n, int W, cudaStream_t st)
{
    pack_input_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, c, d, e, x, n, W);
    return cudaGetLastError();
}

cudaError_t launch_tconv_fwd(int ci, int co, const __nv_bfloat16 *in, const float *K, const float *bias,
                             __nv_bfloat16 *out, int Hi, int Wi, int B, cudaStream_t st)
{
    const size_t n = (size_t)B * Hi * Wi;
    const unsigned g = (unsigned)((n + 255) / 256);
    if (ci == 32 && co == 32) tconv_fwd_kernel<32, 32><<<g, 256, 0, st>>>(in, K, bias, out, Hi, Wi, B);
    else if (ci == 16 && co == 16) tconv_fwd_kernel<16, 16><<<g, 256, 0, st>>>(in, K, bias, out, Hi, Wi, B);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// pixels per block of the transposed-conv backward (static shared memory < 48 KB)
static int tconv_bwd_px(int ci) { return ci == 32 ? 64 : 128; }

// Blocks of the transposed-conv backward (and partial rows it writes): one
// per chunk of input pixels up to 8 per SM of a 148-SM part.
constexpr size_t kTconvMaxBlocks = 1184;
size_t tconv_blocks(int ci, int Hi, int Wi, int B)
{
    const int k = tconv_bwd_px(ci);
    const size_t chunks = ((size_t)B * Hi * Wi + k - 1) / k;
    return chunks < kTconvMaxBlocks ? chunks : kTconvMaxBlocks;
}

cudaError_t launch_tconv_bwd(int ci, int co, const __nv_bfloat16 *in, const __nv_bfloat16 *dout, const float *K,
                             __nv_bfloat16 *dz_in, float *partial, int Hi, int Wi, int B, cudaStream_t st)
{
    const unsigned g = (unsigned)tconv_blocks(ci, Hi, Wi, B);
    if (ci == 32 && co == 32) tconv_bwd_kernel<32, 32, 64><<<g, 64, 0, st>>>(in, dout, K, dz_in, partial, Hi, Wi, B);
    else if (ci == 16 && co == 16)
        tconv_bwd_kernel<16, 16, 128><<<g, 128, 0, st>>>(in, dout, K, dz_in, partial, Hi, Wi, B);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_head_fwd(const __nv_bfloat16 *x, const float *K, const float *bias, float *band, float *alpha,
                            size_t n, cudaStream_t st)
{
    head_fwd_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, K, bias, band, alpha, n);
    return cudaGetLastError();
}

size_t head_blocks(size_t n)
{
    const size_t g = (n + kHeadThreads - 1) / kHeadThreads;
    return g < (size_t)kHeadMaxBlocks ? g : (size_t)kHeadMaxBlocks;
}

cudaError_t launch_head_bwd(const __nv_bfloat16 *x, const float *K, const float *bias, const float *gband,
                            const float *galpha, __nv_bfloat16 *dz, float *partial, size_t n, cudaStream_t st)
{
    head_bwd_kernel<<<(unsigned)head_blocks(n), kHeadThreads, 0, st>>>(x, K, bias, gband, galpha, dz, partial, n);
    return cudaGetLastError();
}

cudaError_t launch_pool_bwd(int C, const __nv_bfloat16 *act, const __nv_bfloat16 *pooled,
                            const __nv_bfloat16 *dpool, const __nv_bfloat16 *dskip, __nv_bfloat16 *dz, int H, int W,
                            int B, cudaStream_t st)
{
    if ((H | W) & 1) return cudaErrorInvalidValue;   // the network's levels are even-sized
    const size_t n = (size_t)B * (H / 2) * (W / 2);
    const unsigned g = (unsigned)((n + 255) / 256);
    if (C == 8) pool_bwd_kernel<8><<<g, 256, 0, st>>>(act, pooled, dpool, dskip, dz, H, W, B);
    else if (C == 16) pool_bwd_kernel<16><<<g, 256, 0, st>>>(act, pooled, dpool, dskip, dz, H, W, B);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

size_t reduce_floats(int n, int tiles) { return (size_t)n * tiles; }

cudaError_t launch_reduce(float *partial, float *out, int n, int tiles, cudaStream_t st)
{
    reduce_kernel<<<(n + 31) / 32, 32 * kReduceWarps, 0, st>>>(partial, out, n, tiles);
    return cudaGetLastError();
}

cudaError_t launch_adam(float *w, const float *g, float *m, float *v, int n, int *step, float lr, float b1, float b2,
                        float eps, cudaStream_t st)
{
    adam_kernel<<<(n + 255) / 256, 256, 0, st>>>(w, g, m, v, n, step, lr, b1, b2, eps);
    step_kernel<<<1, 1, 0, st>>>(step);
    return cudaGetLastError();
}

}  // namespace unet
}  // namespace cd
