// Window sweep shared by the spatial-filter kernels (forward, band gradient,
// fused filter + aggregation loss).
//
// Buffers A and B share every tap: the same albedo / normal / pixel
// distances and the same tile pixel, with their own colours, weights and
// sums.  The sweep therefore keeps A and B side by side in 64-bit register
// pairs and does their arithmetic with Blackwell's packed FP32x2
// instructions (fma/mul/add/sub .rn.f32x2): one instruction for both
// buffers, the same IEEE rounding per lane as the scalar code, so the sums
// are bit-identical to the scalar kernels and to the reference.  The FMA
// pipe executes a pair in two cycles, so the gain is issue bandwidth: the
// sweep becomes FMA-pipe bound instead of issue bound.
//
// Tile layout (shared memory): per pixel three 16-byte records
//   r0 = (A.x, B.x | A.y, B.y)   r1 = (A.z, B.z | alb.x, n.x)
//   r2 = (alb.y, n.y | alb.z, n.z)
// so every pair the sweep needs is one 64-bit half of a record.  A warp
// reads 32 consecutive pixels: per quarter warp 8 records 48 B apart, which
// fall in 8 distinct 4-bank groups (conflict free).
#pragma once
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "f32x2.cuh"

namespace cd {
namespace fsw {

using x2::f2;   // two floats: low half = buffer A, high half = buffer B
using x2::pack;
using x2::lo;
using x2::hi;
using x2::fma2;
using x2::mul2;
using x2::add2;
using x2::sub2;
using x2::sqnorm2;

constexpr int kBX = 32, kBY = 8;

struct Geom {
    int hw, tw, th;
};

CD_DEV Geom geom(int hw) { return Geom{hw, kBX + 2 * hw, kBY + 2 * hw}; }

// bytes of shared memory: three records per tile pixel + the (pd, pd) table
__host__ __device__ inline size_t smem_bytes(int hw)
{
    const int tw = kBX + 2 * hw, th = kBY + 2 * hw, w = 2 * hw + 1;
    return (size_t)3 * tw * th * 16 + (size_t)w * w * 8;
}

// Stage the CTA's footprint (reflect-101, clamped past the reflect range,
// which only pixels outside the image reach) and the table
// pd(ky, kx) = (dx/r)^2 + (dy/r)^2 with (dx, dy) = ((hw-kx)/r, (hw-ky)/r),
// rounded as the reference's dx*dx + dy*dy.
CD_DEV void stage(ulonglong2 *tile, f2 *pdtab, const float *ia, const float *ib, const float *al,
                  const float *nr, int H, int W, int hw)
{
    const int tw = kBX + 2 * hw, th = kBY + 2 * hw;
    const int x0 = blockIdx.x * kBX - hw, y0 = blockIdx.y * kBY - hw;
    const int tid = threadIdx.y * kBX + threadIdx.x;
    for (int t = tid; t < tw * th; t += kBX * kBY) {
        const int ty = t / tw, tx = t - ty * tw;
        const int gx = min(max(mirror(x0 + tx, W), 0), W - 1);
        const int gy = min(max(mirror(y0 + ty, H), 0), H - 1);
        const size_t q = (size_t)gy * W + gx;
        const float3 a = ld3(ia, q), b = ld3(ib, q), l = ld3(al, q), n = ld3(nr, q);
        tile[3 * t + 0] = make_ulonglong2(pack(a.x, b.x), pack(a.y, b.y));
        tile[3 * t + 1] = make_ulonglong2(pack(a.z, b.z), pack(l.x, n.x));
        tile[3 * t + 2] = make_ulonglong2(pack(l.y, n.y), pack(l.z, n.z));
    }
    const int w = 2 * hw + 1;
    for (int k = tid; k < w * w; k += kBX * kBY) {
        const int ky = k / w, kx = k - ky * w;
        const float dy = (float)(hw - ky) / (float)hw, dx = (float)(hw - kx) / (float)hw;
        // dx * dx + dy * dy as the reference's compiled loop rounds it: dy * dy
        // (outer loop) is hoisted and rounded, dx * dx is fused into the add
        const float pd = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
        pdtab[k] = pack(pd, pd);
    }
}

// Per-pixel constants of the sweep.
struct Centre {
    f2 ab_x, ab_y, ab_z;        // (A, B) colour of the pixel
    f2 an_x, an_y, an_z;        // (albedo, normal) of the pixel
    f2 nb01, nb2, nb3, nb4;     // (-band0, -band1), (-band2, -band2), ...
};

// Sums accumulated over the window.
//   acc: (accA, accB) per channel and (wsumA, wsumB)
//   par: band partials P_k = sum_t w d_k [col, 1] (positive; the reference's
//        partials are their negation), k = 0 colour, 1 albedo, 2 normal,
//        3 pixel distance
struct Sums {
    f2 acc_x, acc_y, acc_z, acc_w;
    f2 px[4], py[4], pz[4], pw[4];
};

// How the sweep evaluates a tap's weight exp(e), e <= 0:
//   kExpf     __expf, as the reference's kernel (ops/regression.cu.cc:149-150)
//   kExp2Ftz  2^(e * log2(e)) on the ex2.approx.ftz instruction: the same
//             values wherever exp(e) is a normal float, zero below 2^-126
//             (measured 6 % faster on the fused 11x11 sweep at 1080p)
constexpr int kExpf = 0, kExp2Ftz = 1;

template <int kExp>
CD_DEV float weight_exp(float e)
{
    if (kExp == kExp2Ftz) {
        float y;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(e * 1.44269504088896341f));
        return y;
    }
    return __expf(e);
}

template <bool kAcc, bool kPar, int kExp = kExpf>
CD_DEV void tap(const ulonglong2 *rec, f2 pd2, const Centre &c, Sums &s)
{
    const ulonglong2 r0 = rec[0], r1 = rec[1], r2 = rec[2];
    // colour differences of both buffers, albedo/normal differences
    const f2 dab_x = sub2(c.ab_x, r0.x), dab_y = sub2(c.ab_y, r0.y), dab_z = sub2(c.ab_z, r1.x);
    const f2 dan_x = sub2(c.an_x, r1.y), dan_y = sub2(c.an_y, r2.x), dan_z = sub2(c.an_z, r2.y);
    const f2 dAB = sqnorm2(dab_x, dab_y, dab_z);            // (|dA|^2, |dB|^2)
    const f2 dAN = sqnorm2(dan_x, dan_y, dan_z);            // (|dalb|^2, |dn|^2)
    const float dal = lo(dAN), dn = hi(dAN);
    const f2 dal2 = pack(dal, dal), dn2 = pack(dn, dn);
    // e = ((-b0*dA - b2*dAl) - b3*dN) - b4*pd (ops/regression.cu.cc:147-148)
    // rounded as the compiled reference: the first product fused with the
    // rounded second, the later products fused into the running sum
    const f2 e = fma2(c.nb4, pd2, fma2(c.nb3, dn2, fma2(c.nb01, dAB, mul2(c.nb2, dal2))));
    const f2 w = pack(weight_exp<kExp>(lo(e)), weight_exp<kExp>(hi(e)));
    if (kAcc) {
        const f2 col_x = r0.x, col_y = r0.y, col_z = r1.x;
        s.acc_x = fma2(w, col_x, s.acc_x);
        s.acc_y = fma2(w, col_y, s.acc_y);
        s.acc_z = fma2(w, col_z, s.acc_z);
        s.acc_w = add2(s.acc_w, w);
    }
    if (kPar) {
        const f2 dk[4] = {dAB, dal2, dn2, pd2};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const f2 dw = mul2(w, dk[k]);
            s.px[k] = fma2(dw, r0.x, s.px[k]);
            s.py[k] = fma2(dw, r0.y, s.py[k]);
            s.pz[k] = fma2(dw, r1.x, s.pz[k]);
            s.pw[k] = add2(s.pw[k], dw);
        }
    }
}

// Sweep the (2hw+1)^2 window of the thread's pixel.  HW > 0 fixes the
// radius at compile time (fully unrolled rows); HW == 0 takes it at run time.
template <int HW, bool kAcc, bool kPar, int kExp = kExpf>
CD_DEV void sweep(const ulonglong2 *tile, const f2 *pdtab, int hw_rt, const Centre &c, Sums &s)
{
    const int hw = HW > 0 ? HW : hw_rt;
    const int tw = kBX + 2 * hw, w = 2 * hw + 1;
    for (int ky = 0; ky < w; ++ky) {
        const ulonglong2 *row = tile + 3 * ((threadIdx.y + ky) * tw + threadIdx.x);
        const f2 *pdrow = pdtab + ky * w;
        if (HW > 0) {
#pragma unroll
            for (int kx = 0; kx < 2 * HW + 1; ++kx) tap<kAcc, kPar, kExp>(row + 3 * kx, pdrow[kx], c, s);
        } else {
            for (int kx = 0; kx < w; ++kx) tap<kAcc, kPar, kExp>(row + 3 * kx, pdrow[kx], c, s);
        }
    }
}

CD_DEV Centre centre(const ulonglong2 *tile, int hw, const float *band5)
{
    const int tw = kBX + 2 * hw;
    const ulonglong2 *r = tile + 3 * ((threadIdx.y + hw) * tw + threadIdx.x + hw);
    Centre c;
    c.ab_x = r[0].x;
    c.ab_y = r[0].y;
    c.ab_z = r[1].x;
    c.an_x = r[1].y;
    c.an_y = r[2].x;
    c.an_z = r[2].y;
    const float b0 = __ldg(band5), b1 = __ldg(band5 + 1), b2 = __ldg(band5 + 2);
    const float b3 = __ldg(band5 + 3), b4 = __ldg(band5 + 4);
    c.nb01 = pack(-b0, -b1);
    c.nb2 = pack(-b2, -b2);
    c.nb3 = pack(-b3, -b3);
    c.nb4 = pack(-b4, -b4);
    return c;
}

CD_DEV void zero(Sums &s)
{
    const f2 z = pack(0.f, 0.f);
    s.acc_x = s.acc_y = s.acc_z = s.acc_w = z;
#pragma unroll
    for (int k = 0; k < 4; ++k) s.px[k] = s.py[k] = s.pz[k] = s.pw[k] = z;
}

// dL/dband from the partials and the upstream gradient of the four filter
// outputs, as SpatialFilterGradKernel (ops/regression.cu.cc:64-80) forms it:
// band0 <- A only, band1 <- B only, band2..4 <- A + B.  The reference's
// partials are -P_k, so each dot product is negated.
CD_DEV void band_grad(const Sums &s, float3 gA, float3 gB, float gwA, float gwB, float *o)
{
    float oA[4], oB[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        oA[k] = -fmaf(gwA, lo(s.pw[k]), fmaf(gA.z, lo(s.pz[k]), fmaf(gA.x, lo(s.px[k]), gA.y * lo(s.py[k]))));
        oB[k] = -fmaf(gwB, hi(s.pw[k]), fmaf(gB.z, hi(s.pz[k]), fmaf(gB.x, hi(s.px[k]), gB.y * hi(s.py[k]))));
    }
    o[0] = oA[0];
    o[1] = oB[0];
    o[2] = oA[1] + oB[1];
    o[3] = oA[2] + oB[2];
    o[4] = oA[3] + oB[3];
}

}  // namespace fsw
}  // namespace cd
