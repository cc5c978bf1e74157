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
//
// Fused erosion + screening with a one-pixel history window (win_prev = 1,
// the reference's setting) runs as a persistent kernel: each CTA walks the
// 32x8 tiles with stride gridDim.x, and the next two tiles' inputs (both
// colour footprints with the window's halo, the three history buffers and
// the raw mask with a one-pixel halo) arrive by TMA into a double buffer
// while the current tile computes, so the DRAM latency is off the critical
// path.  Its row pass slides the window over four output columns per
// (channel, row, column group) item, in registers, on all threads.  Other window sizes and images whose rows are not a multiple
// of 16 bytes take the tile-per-CTA kernel above it.
#include <atomic>
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "tma.cuh"

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


// ---------------------------------------------------------------------------
// Persistent TMA kernel (fused erosion, win_prev = 1, HC = win_curr / 2).
// ---------------------------------------------------------------------------
struct TsMaps {
    CUtensorMap c1, c2, h0, h1, h2, mk;   // current1/2 and prev/prev1/prev2 as (3W, H, B) floats; mask (W, H, B) bytes
};

template <int HC>
struct TsGeom {
    static constexpr int TW = kTX + 2 * HC, TH = kTY + 2 * HC;
    // colour box: 3 floats per pixel, the start rounded down to 16 bytes;
    // OFF = the footprint's first float within the box row
    static constexpr int OFF = (4 - (3 * HC) % 4) % 4;
    static constexpr int BOXC = (3 * TW + OFF + 3) & ~3;
    static constexpr int CBYTES = ((TH * BOXC * 4 + 127) / 128) * 128;
    static constexpr int HBOX = 3 * kTX;                 // history box: the tile's 32 pixels
    static constexpr int HBYTES = kTY * HBOX * 4;
    static constexpr int MBOXX = 64, MBOXY = kTY + 2;    // mask box: columns x0-16 .. x0+47, rows y0-1 .. y0+8
    static constexpr int MBYTES = MBOXX * MBOXY;
    static constexpr int STAGE = 2 * CBYTES + 3 * HBYTES + MBYTES;
    static constexpr int TX_BYTES = 2 * TH * BOXC * 4 + 3 * HBYTES + MBYTES;
    static constexpr int PLANES = 2 * kVals * TH * kTX * 4;   // row-pass minima and maxima
    static constexpr int SMEM = 2 * STAGE + PLANES + 16;
    static constexpr int NJ = 4 + 2 * HC;                  // input columns of a 4-output row segment
};

__device__ int g_image_kernel_error = 0;   // sticky: bit 0 = a temporal-screening staging wait ran out

constexpr int kWaitPolls = 1 << 22;

// min and max over the 2*HC+1 consecutive values starting at each of 4
// positions of a[0 .. 4 + 2*HC); NaN (out-of-image) values are skipped.
template <int HC>
CD_DEV void window4(const float *a, float *mn, float *mx)
{
    if constexpr (HC == 3) {
        float n2[9], x2[9], n4[7], x4[7];
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            n2[i] = fminf(a[i], a[i + 1]);
            x2[i] = fmaxf(a[i], a[i + 1]);
        }
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            n4[i] = fminf(n2[i], n2[i + 2]);
            x4[i] = fmaxf(x2[i], x2[i + 2]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            mn[i] = fminf(n4[i], n4[i + 3]);
            mx[i] = fmaxf(x4[i], x4[i + 3]);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float n = a[i], x = a[i];
#pragma unroll
            for (int d = 1; d <= 2 * HC; ++d) {
                n = fminf(n, a[i + d]);
                x = fmaxf(x, a[i + d]);
            }
            mn[i] = n;
            mx[i] = x;
        }
    }
}

template <int HC>
__global__ void __launch_bounds__(kTX * kTY, 2) temporal_tma_kernel(
    const __grid_constant__ TsMaps maps, float *__restrict__ eroded, float *__restrict__ out,
    float *__restrict__ out1, float *__restrict__ out2, float *__restrict__ succ, int H, int W, int ntx,
    int nty, int ntiles)
{
    using G = TsGeom<HC>;
    extern __shared__ __align__(128) unsigned char smem[];
    float *rmin = reinterpret_cast<float *>(smem + 2 * G::STAGE);
    float *rmax = rmin + kVals * G::TH * kTX;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * G::STAGE + G::PLANES);
    const int tid = threadIdx.y * kTX + threadIdx.x;
    const int per_img = ntx * nty;
    const float qnan = __int_as_float(0x7fffffff);

    auto issue = [&](int t, int s) {
        const int b = t / per_img, r = t - b * per_img, by = r / ntx, bx = r - by * ntx;
        unsigned char *st = smem + s * G::STAGE;
        tc::mbar_expect_tx(&bar[s], G::TX_BYTES);
        const int xc = tma::floor_to(3 * (bx * kTX - HC), 4), yc = by * kTY - HC;
        tma::load3(st, &maps.c1, xc, yc, b, &bar[s]);
        tma::load3(st + G::CBYTES, &maps.c2, xc, yc, b, &bar[s]);
        unsigned char *hs = st + 2 * G::CBYTES;
        tma::load3(hs, &maps.h0, 3 * kTX * bx, by * kTY, b, &bar[s]);
        tma::load3(hs + G::HBYTES, &maps.h1, 3 * kTX * bx, by * kTY, b, &bar[s]);
        tma::load3(hs + 2 * G::HBYTES, &maps.h2, 3 * kTX * bx, by * kTY, b, &bar[s]);
        tma::load3(hs + 3 * G::HBYTES, &maps.mk, bx * kTX - 16, by * kTY - 1, b, &bar[s]);
    };

    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
    }
    __syncthreads();
    const int G0 = (int)gridDim.x;
    if (tid == 0) {
        if ((int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
        if ((int)blockIdx.x + G0 < ntiles) issue(blockIdx.x + G0, 1);
    }
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += G0, ++it) {
        const int s = it & 1;
        // this barrier also marks every thread done with the previous tile:
        // its stage (and the row planes) may be reused from here on
        const bool landed = __syncthreads_and(tc::mbar_wait(&bar[s], (uint32_t)(it >> 1) & 1u, kWaitPolls)) != 0;
        if (landed && it >= 1 && tid == 0 && t + G0 < ntiles) issue(t + G0, s ^ 1);
        if (!landed) {
            // the other stage has a copy in flight only on the first tile
            // (the prologue's second copy; later ones are issued after a
            // landed wait): give it a bounded wait, and report the time-out
            if (tid == 0) {
                atomicOr(&g_image_kernel_error, 1);
                if (it == 0 && t + G0 < ntiles) tc::mbar_wait(&bar[1], 0u, kWaitPolls);
            }
            return;
        }
        const int b = t / per_img, rr = t - b * per_img, by = rr / ntx, bx = rr - by * ntx;
        const size_t px = (size_t)H * W;
        const float *C1 = reinterpret_cast<const float *>(smem + s * G::STAGE);
        const float *C2 = reinterpret_cast<const float *>(smem + s * G::STAGE + G::CBYTES);
        const float *H0 = reinterpret_cast<const float *>(smem + s * G::STAGE + 2 * G::CBYTES);
        const float *H1 = H0 + kTY * G::HBOX, *H2 = H1 + kTY * G::HBOX;
        const unsigned char *MK = smem + s * G::STAGE + 2 * G::CBYTES + 3 * G::HBYTES;

        // row pass: item (c, r, q) = channel c, tile row r, output columns
        // 4q .. 4q + 3: the channel's current1 and current2 values of the
        // segment are loaded once and give all three quantities (current1,
        // current2, their average); 3 * TH * 8 items over all threads
        for (int it = tid; it < 3 * G::TH * 8; it += kTX * kTY) {
            const int q = it & 7, rc = it >> 3, c = rc % 3, r = rc / 3;
            const int gy = by * kTY - HC + r;
            const int gx0 = bx * kTX - HC + 4 * q;
            const bool row_in = gy >= 0 && gy < H;
            const bool all_in = row_in && gx0 >= 0 && gx0 + G::NJ <= W;
            const int o = r * G::BOXC + G::OFF + 12 * q + c;
            float a[G::NJ], bb[G::NJ], v[G::NJ];
#pragma unroll
            for (int j = 0; j < G::NJ; ++j) {
                const bool in = all_in || (row_in && gx0 + j >= 0 && gx0 + j < W);
                a[j] = in ? C1[o + 3 * j] : qnan;
                bb[j] = in ? C2[o + 3 * j] : qnan;
                v[j] = (a[j] + bb[j]) * 0.5f;
            }
            float mn[4], mx[4];
            const int d = r * kTX + 4 * q;
            window4<HC>(a, mn, mx);
            *reinterpret_cast<float4 *>(rmin + c * G::TH * kTX + d) = make_float4(mn[0], mn[1], mn[2], mn[3]);
            *reinterpret_cast<float4 *>(rmax + c * G::TH * kTX + d) = make_float4(mx[0], mx[1], mx[2], mx[3]);
            window4<HC>(bb, mn, mx);
            *reinterpret_cast<float4 *>(rmin + (3 + c) * G::TH * kTX + d) = make_float4(mn[0], mn[1], mn[2], mn[3]);
            *reinterpret_cast<float4 *>(rmax + (3 + c) * G::TH * kTX + d) = make_float4(mx[0], mx[1], mx[2], mx[3]);
            window4<HC>(v, mn, mx);
            *reinterpret_cast<float4 *>(rmin + (6 + c) * G::TH * kTX + d) = make_float4(mn[0], mn[1], mn[2], mn[3]);
            *reinterpret_cast<float4 *>(rmax + (6 + c) * G::TH * kTX + d) = make_float4(mx[0], mx[1], mx[2], mx[3]);
        }
        __syncthreads();

        const int tx = threadIdx.x, ty = threadIdx.y;
        const int cx = bx * kTX + tx, cy = by * kTY + ty;
        if (cx < W && cy < H) {
            const size_t p = b * px + (size_t)cy * W + cx;
            // 3x3 erosion of the raw mask, image pixels only (the TMA fills
            // out-of-image bytes with zeros; the min ignores them)
            bool keep = true;
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    const bool in = cx + dx >= 0 && cx + dx < W && cy + dy >= 0 && cy + dy < H;
                    keep = keep && (!in || MK[(ty + 1 + dy) * G::MBOXX + tx + 16 + dx] != 0);
                }
            const float m = keep ? 1.f : 0.f;
            eroded[p] = m;
            const int co = (ty + HC) * G::BOXC + G::OFF + 3 * (tx + HC);
            const float3 a1 = make_float3(C1[co], C1[co + 1], C1[co + 2]);
            const float3 a2 = make_float3(C2[co], C2[co + 1], C2[co + 2]);
            const float3 cu = make_float3((a1.x + a2.x) * 0.5f, (a1.y + a2.y) * 0.5f, (a1.z + a2.z) * 0.5f);
            if (m + 1e-4f < 1.f) {
                st3(out, p, cu);
                st3(out1, p, a1);
                st3(out2, p, a2);
                succ[p] = 0.f;
            } else {
                float mnC[kVals], mxC[kVals];
#pragma unroll
                for (int k = 0; k < kVals; ++k) {
                    float n = kBig, x = -kBig;
#pragma unroll
                    for (int dy = 0; dy <= 2 * HC; ++dy) {
                        n = fminf(n, rmin[(k * G::TH + ty + dy) * kTX + tx]);
                        x = fmaxf(x, rmax[(k * G::TH + ty + dy) * kTX + tx]);
                    }
                    mnC[k] = n;
                    mxC[k] = x;
                }
                const int ho = ty * G::HBOX + 3 * tx;
                const float3 h0 = make_float3(H0[ho], H0[ho + 1], H0[ho + 2]);
                const float3 h1 = make_float3(H1[ho], H1[ho + 1], H1[ho + 2]);
                const float3 h2 = make_float3(H2[ho], H2[ho + 1], H2[ho + 2]);
                // the history window is the pixel itself (its mask is >= 1 here)
                const float hv[kVals] = {h1.x, h1.y, h1.z, h2.x, h2.y, h2.z, h0.x, h0.y, h0.z};
                bool ok[3];
#pragma unroll
                for (int g = 0; g < 3; ++g) {
                    bool o = true;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float mnP = fminf(kBig, hv[3 * g + k]), mxP = fmaxf(-kBig, hv[3 * g + k]);
                        o = o && (mnP < mxC[3 * g + k]) && (mnC[3 * g + k] < mxP);
                    }
                    ok[g] = o;
                }
                st3(out1, p, ok[0] ? h1 : a1);
                st3(out2, p, ok[1] ? h2 : a2);
                st3(out, p, ok[2] ? h0 : cu);
                succ[p] = ok[2] ? 1.f : 0.f;
            }
        }
    }
}

template <int HC>
cudaError_t launch_temporal_tma(const float *c1, const float *c2, const float *prev, const float *prev1,
                                const float *prev2, const uint8_t *raw, float *eroded, float *out, float *out1,
                                float *out2, float *succ, int B, int H, int W, cudaStream_t st, bool *done)
{
    using G = TsGeom<HC>;
    *done = false;
    TsMaps m;
    if (!tma::encode_image(&m.c1, c1, false, 3, W, H, B, G::BOXC, G::TH) ||
        !tma::encode_image(&m.c2, c2, false, 3, W, H, B, G::BOXC, G::TH) ||
        !tma::encode_image(&m.h0, prev, false, 3, W, H, B, G::HBOX, kTY) ||
        !tma::encode_image(&m.h1, prev1, false, 3, W, H, B, G::HBOX, kTY) ||
        !tma::encode_image(&m.h2, prev2, false, 3, W, H, B, G::HBOX, kTY) ||
        !tma::encode_image(&m.mk, raw, true, 1, W, H, B, G::MBOXX, G::MBOXY))
        return cudaSuccess;   // not eligible: the caller takes the tile-per-CTA kernel
    // per-process caches (every thread computes the same values)
    static std::atomic<int> occ_cache{0};
    static std::atomic<int> sm_cache[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(temporal_tma_kernel<HC>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM)) !=
        cudaSuccess)
        return e;
    int occ = occ_cache.load(std::memory_order_relaxed);
    if (!occ) {
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, temporal_tma_kernel<HC>, kTX * kTY, G::SMEM)) !=
            cudaSuccess)
            return e;
        if (occ < 1) return cudaSuccess;
        occ_cache.store(occ, std::memory_order_relaxed);
    }
    int nsm = dev < 64 ? sm_cache[dev].load(std::memory_order_relaxed) : 0;
    if (!nsm) {
        if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if (dev < 64) sm_cache[dev].store(nsm, std::memory_order_relaxed);
    }
    const int ntx = (W + kTX - 1) / kTX, nty = (H + kTY - 1) / kTY, ntiles = ntx * nty * B;
    const int grid = min(ntiles, nsm * occ);
    temporal_tma_kernel<HC><<<grid, dim3(kTX, kTY), G::SMEM, st>>>(m, eroded, out, out1, out2, succ, H, W, ntx, nty,
                                                                   ntiles);
    *done = true;
    return cudaGetLastError();
}

}  // namespace

int temporal_error_flag()
{
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_image_kernel_error, sizeof(int)) != cudaSuccess) return -1;
    return v;
}

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
    if (raw && hp == 0 && hc >= 1 && hc <= 3 && tma::persistent_enabled()) {
        bool done = false;
        e = hc == 3 ? launch_temporal_tma<3>(c1, c2, prev, prev1, prev2, raw, eroded, out, out1, out2, succ, B, H, W,
                                             st, &done)
          : hc == 2 ? launch_temporal_tma<2>(c1, c2, prev, prev1, prev2, raw, eroded, out, out1, out2, succ, B, H, W,
                                             st, &done)
                    : launch_temporal_tma<1>(c1, c2, prev, prev1, prev2, raw, eroded, out, out1, out2, succ, B, H, W,
                                             st, &done);
        if (e != cudaSuccess || done) return e;
    }
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
