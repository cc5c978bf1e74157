// Reprojection-mask erosion and temporal screening on sm_100a.
//
// Reference semantics: tf.nn.erosion2d on the float success mask
// (scripts/main.py:270-276) and the TemporalScreening kernel,
// ops/temporal.cu.cc:28-198.  Temporal screening keeps the reprojected
// history (prev, prev1, prev2) of a pixel when, channel by channel, the
// min/max range of the current window (win_curr, in-bounds taps only)
// overlaps strictly with the min/max range of the history window (win_prev,
// only taps whose eroded mask is >= 1); a pixel whose eroded mask is below 1
// keeps the current values.  Minima and maxima start from the reference's
// +-1e7 sentinel (ops/temporal.cu.cc:29).
//
// The current window is evaluated separably: a row pass over a shared-memory
// tile (32x8 pixels plus the radius) takes the min/max along x, a column pass
// along y.  Out-of-image taps are stored as NaN, which fminf/fmaxf skip, so
// the result equals the reference's in-bounds loop.  The accept/reject
// decisions are exact: they involve only additions, halvings and compares.
#include <cuda_runtime.h>
#include "cd_common.cuh"

namespace cd {
namespace {

constexpr int kTX = 32, kTY = 8;
constexpr float kBig = 10000000.f;
constexpr int kVals = 9;   // current1.xyz, current2.xyz, (current1+current2)/2 .xyz

// tile planes (6 x tw x th floats), row-pass planes (2 x kVals x th x kTX
// floats) and the raw mask footprint ((kTX + 2 + 2hp) x (kTY + 2 + 2hp) bytes)
__host__ __device__ inline size_t ts_smem(int hc, int hp)
{
    const int tw = kTX + 2 * hc, th = kTY + 2 * hc;
    return ((size_t)6 * tw * th + (size_t)2 * kVals * th * kTX) * sizeof(float) +
           (size_t)(kTX + 2 + 2 * hp) * (kTY + 2 + 2 * hp);
}

// min over the in-bounds 3x3 window of the byte mask, as 0.f / 1.f
CD_DEV float eroded_at(const uint8_t *mask, int x, int y, int H, int W)
{
    float m = 1.f;
    for (int yy = max(0, y - 1); yy <= min(H - 1, y + 1); ++yy)
        for (int xx = max(0, x - 1); xx <= min(W - 1, x + 1); ++xx)
            m = fminf(m, __ldg(mask + (size_t)yy * W + xx) ? 1.f : 0.f);
    return m;
}

__global__ void __launch_bounds__(256) erode_kernel(const uint8_t *__restrict__ mask,
                                                    float *__restrict__ out, int H, int W)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t base = (size_t)blockIdx.z * H * W;
    out[base + (size_t)y * W + x] = eroded_at(mask + base, x, y, H, W);
}

template <bool kFused>
__global__ void __launch_bounds__(kTX * kTY, 3) temporal_kernel(
    const float *__restrict__ cur1, const float *__restrict__ cur2,
    const float *__restrict__ prev, const float *__restrict__ prev1,
    const float *__restrict__ prev2, const float *__restrict__ rs,
    const uint8_t *__restrict__ raw, float *__restrict__ eroded, float *__restrict__ out,
    float *__restrict__ out1, float *__restrict__ out2, float *__restrict__ succ, int H, int W,
    int hc, int hp)
{
    extern __shared__ float sm[];
    const int tw = kTX + 2 * hc, th = kTY + 2 * hc;
    const int tplane = tw * th, rplane = th * kTX;
    float *tile = sm;                       // 6 planes: c1.xyz, c2.xyz
    float *rmin = sm + 6 * tplane;          // kVals planes [th][kTX]
    float *rmax = rmin + kVals * rplane;

    const size_t px = (size_t)H * W, b = blockIdx.z;
    cur1 += 3 * px * b;
    cur2 += 3 * px * b;
    prev += 3 * px * b;
    prev1 += 3 * px * b;
    prev2 += 3 * px * b;
    if (kFused) {
        raw += px * b;
        eroded += px * b;
    } else {
        rs += px * b;
    }
    out += 3 * px * b;
    out1 += 3 * px * b;
    out2 += 3 * px * b;
    succ += px * b;

    uint8_t *smask = reinterpret_cast<uint8_t *>(rmax + kVals * rplane);
    const int tid = threadIdx.y * kTX + threadIdx.x;
    const int x0 = blockIdx.x * kTX - hc, y0 = blockIdx.y * kTY - hc;
    const float qnan = __int_as_float(0x7fffffff);
    // The pixel's history does not depend on the tile: issue its loads first
    // so their latency overlaps the staging and the row pass.
    const int cx = blockIdx.x * kTX + threadIdx.x, cy = blockIdx.y * kTY + threadIdx.y;
    const bool inside = cx < W && cy < H;
    const size_t p = inside ? (size_t)cy * W + cx : 0;
    const float3 h0 = ld3(prev, p), h1 = ld3(prev1, p), h2 = ld3(prev2, p);
    // current-frame footprint, as planes
    for (int t = tid; t < tplane; t += kTX * kTY) {
        const int ty = t / tw, tx = t - ty * tw;
        const int gx = x0 + tx, gy = y0 + ty;
        float3 a = make_float3(qnan, qnan, qnan), c = a;   // outside the image: skipped by fminf / fmaxf
        if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
            a = ld3(cur1, (size_t)gy * W + gx);
            c = ld3(cur2, (size_t)gy * W + gx);
        }
        tile[0 * tplane + t] = a.x;
        tile[1 * tplane + t] = a.y;
        tile[2 * tplane + t] = a.z;
        tile[3 * tplane + t] = c.x;
        tile[4 * tplane + t] = c.y;
        tile[5 * tplane + t] = c.z;
    }
    // raw mask footprint for the erosion of every pixel within hp of the
    // tile; outside the image 1, which the min ignores
    const int mw = kTX + 2 + 2 * hp, mh = kTY + 2 + 2 * hp;
    const int mx0 = blockIdx.x * kTX - 1 - hp, my0 = blockIdx.y * kTY - 1 - hp;
    if (kFused) {
        for (int i = tid; i < mw * mh; i += kTX * kTY) {
            const int r = i / mw, q = i - r * mw, gx = mx0 + q, gy = my0 + r;
            smask[i] = gx >= 0 && gx < W && gy >= 0 && gy < H ? (__ldg(raw + (size_t)gy * W + gx) ? 1 : 0) : 1;
        }
    }
    __syncthreads();
    // eroded mask at image pixel (x, y), |x - cx| <= hp, |y - cy| <= hp
    auto eroded_s = [&](int x, int y) {
        const uint8_t *r0 = smask + (y - my0 - 1) * mw + (x - mx0 - 1);
        const uint8_t v = r0[0] & r0[1] & r0[2] & r0[mw] & r0[mw + 1] & r0[mw + 2] & r0[2 * mw] & r0[2 * mw + 1] &
                          r0[2 * mw + 2];
        return v ? 1.f : 0.f;
    };
    const float m = inside ? (kFused ? eroded_s(cx, cy) : __ldg(rs + p)) : 0.f;
    // row pass: min/max along x over 2*hc+1 tile columns
    for (int t = tid; t < rplane; t += kTX * kTY) {
        const int r = t / kTX, x = t - r * kTX;
        float mn[kVals], mx[kVals];
#pragma unroll
        for (int k = 0; k < kVals; ++k) {
            mn[k] = kBig;
            mx[k] = -kBig;
        }
        for (int dx = 0; dx <= 2 * hc; ++dx) {
            const int o = r * tw + x + dx;
            float v[kVals];
#pragma unroll
            for (int k = 0; k < 6; ++k) v[k] = tile[k * tplane + o];
#pragma unroll
            for (int k = 0; k < 3; ++k) v[6 + k] = (v[k] + v[3 + k]) * 0.5f;
#pragma unroll
            for (int k = 0; k < kVals; ++k) {
                mn[k] = fminf(mn[k], v[k]);
                mx[k] = fmaxf(mx[k], v[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < kVals; ++k) {
            rmin[k * rplane + t] = mn[k];
            rmax[k * rplane + t] = mx[k];
        }
    }
    __syncthreads();

    if (!inside) return;
    const int co = (threadIdx.y + hc) * tw + threadIdx.x + hc;
    const float3 a1 = make_float3(tile[co], tile[tplane + co], tile[2 * tplane + co]);
    const float3 a2 = make_float3(tile[3 * tplane + co], tile[4 * tplane + co], tile[5 * tplane + co]);
    const float3 cu = make_float3((a1.x + a2.x) * 0.5f, (a1.y + a2.y) * 0.5f, (a1.z + a2.z) * 0.5f);
    if (kFused) eroded[p] = m;
    if (m + 1e-4f < 1.f) {
        st3(out, p, cu);
        st3(out1, p, a1);
        st3(out2, p, a2);
        succ[p] = 0.f;
        return;
    }
    // column pass for the current window
    float mnC[kVals], mxC[kVals];
#pragma unroll
    for (int k = 0; k < kVals; ++k) {
        mnC[k] = kBig;
        mxC[k] = -kBig;
    }
    for (int dy = 0; dy <= 2 * hc; ++dy) {
        const int o = (threadIdx.y + dy) * kTX + threadIdx.x;
#pragma unroll
        for (int k = 0; k < kVals; ++k) {
            mnC[k] = fminf(mnC[k], rmin[k * rplane + o]);
            mxC[k] = fmaxf(mxC[k], rmax[k * rplane + o]);
        }
    }
    // history window: prev, prev1, prev2 at taps whose mask is >= 1
    float mnP[kVals], mxP[kVals];
#pragma unroll
    for (int k = 0; k < kVals; ++k) {
        mnP[k] = kBig;
        mxP[k] = -kBig;
    }
    for (int iy = cy - hp; iy <= cy + hp; ++iy)
        for (int ix = cx - hp; ix <= cx + hp; ++ix) {
            if (ix < 0 || ix >= W || iy < 0 || iy >= H) continue;
            const size_t q = (size_t)iy * W + ix;
            const bool centre = ix == cx && iy == cy;
            const float mq = centre ? m : (kFused ? eroded_s(ix, iy) : __ldg(rs + q));
            if (mq < 1.f) continue;
            const float3 v0 = centre ? h0 : ld3(prev, q), v1 = centre ? h1 : ld3(prev1, q);
            const float3 v2 = centre ? h2 : ld3(prev2, q);
            const float v[kVals] = {v1.x, v1.y, v1.z, v2.x, v2.y, v2.z, v0.x, v0.y, v0.z};
#pragma unroll
            for (int k = 0; k < kVals; ++k) {
                mnP[k] = fminf(mnP[k], v[k]);
                mxP[k] = fmaxf(mxP[k], v[k]);
            }
        }
    // value slots: 0..2 -> pair 1, 3..5 -> pair 2, 6..8 -> averaged pair
    bool ok[3];
#pragma unroll
    for (int g = 0; g < 3; ++g) {
        bool o = true;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            o = o && (mnP[3 * g + k] < mxC[3 * g + k]) && (mnC[3 * g + k] < mxP[3 * g + k]);
        ok[g] = o;
    }
    st3(out1, p, ok[0] ? h1 : a1);
    st3(out2, p, ok[1] ? h2 : a2);
    st3(out, p, ok[2] ? h0 : cu);
    succ[p] = ok[2] ? 1.f : 0.f;
}

}  // namespace

cudaError_t launch_erode3x3(const uint8_t *mask, float *out, int B, int H, int W, cudaStream_t st)
{
    dim3 block(32, 8);
    dim3 grid((W + 31) / 32, (H + 7) / 8, B);
    erode_kernel<<<grid, block, 0, st>>>(mask, out, H, W);
    return cudaGetLastError();
}

cudaError_t launch_temporal(const float *c1, const float *c2, const float *prev,
                            const float *prev1, const float *prev2, const float *rs,
                            const uint8_t *raw, float *eroded, float *out, float *out1,
                            float *out2, float *succ, int B, int H, int W, int win_curr,
                            int win_prev, cudaStream_t st)
{
    const int hc = win_curr / 2, hp = win_prev / 2;
    const size_t smem = ts_smem(hc, hp);
    if (smem > 220 * 1024) return cudaErrorInvalidConfiguration;
    dim3 block(kTX, kTY);
    dim3 grid((W + kTX - 1) / kTX, (H + kTY - 1) / kTY, B);
    cudaError_t e;
    if (raw) {
        e = cudaFuncSetAttribute(temporal_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return e;
        temporal_kernel<true><<<grid, block, smem, st>>>(c1, c2, prev, prev1, prev2, nullptr, raw,
                                                         eroded, out, out1, out2, succ, H, W, hc, hp);
    } else {
        e = cudaFuncSetAttribute(temporal_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return e;
        temporal_kernel<false><<<grid, block, smem, st>>>(c1, c2, prev, prev1, prev2, rs, nullptr,
                                                          nullptr, out, out1, out2, succ, H, W, hc, hp);
    }
    return cudaGetLastError();
}

}  // namespace cd
