// SVGF-style backward reprojection on sm_100a.
//
// Reference semantics: isReprojValid + Reproject, ops/reproject.cu.cc:32-238.
// Per pixel: reject if opacity == 0; otherwise test the four bilinear taps
// around floor(pos) + mvec * dim (truncated to int) for screen border (on the
// rounded position), depth and normal consistency; blend the valid taps with
// renormalised bilinear weights when their weight sum is >= 0.01, else fall
// back to the plain average of the valid taps of a 3x3 box around the rounded
// position.  The success mask is the reference's bit for bit: every float
// expression that decides it is written with explicit rounding intrinsics,
// which the oracle mirrors.  The rounding of each was pinned against the
// reference kernel's own outputs on inputs that sit on the decision
// boundaries: pos + mvec*dim and the squared normal distance are fused
// multiply-adds, the bilinear weight sum adds rounded products.
//
// Unlike the reference, which zeroes the outputs and accumulates into global
// memory through a device-side pointer table uploaded with blocking memcpys
// (ops/reproject.cc:151-153), each thread first decides its taps and weights
// in registers and then writes every output value once; the list of tensors
// travels by value in the kernel parameters.
#include <cuda_runtime.h>
#include "cd_common.cuh"

namespace cd {
namespace {

// Border, depth and normal test (ops/reproject.cu.cc:32-50).  The border
// part is hoisted by the caller (it depends only on the rounded position).
// The normal distance is sqrt(fma(dz,dz, fma(dx,dx, dy*dy))) and its ratio is
// taken in double: the reference adds the double literal 1e-2 (line 46).
//
// Both tests compare a correctly rounded quotient with a constant c whose
// significand is even (10 = 1.25 * 2^3, 4 = 2^2), and they are decided here
// without the division.  Rounding to nearest is monotone and rounds the
// midpoint between c and its successor to c, so for b > 0
//     RN(a / b) > c   <=>   a / b > c + ulp(c) / 2   <=>   a - c b > b ulp(c) / 2.
// Near the threshold a - c b is exact in the working precision: in float,
// a >= 8b makes a a multiple of 8 ulp(b) and 10 b a multiple of 2 ulp(b),
// so their difference, smaller than 2b there, fits 24 bits and the fused
// multiply-add returns it exactly; in double, d and 4 S are within a factor
// of two of each other (Sterbenz), so d - 4 S is exact.  Far from the
// threshold a rounding error cannot move the difference across b ulp(c) / 2.
// The scaled right-hand sides are exact (b >= 2^-100, S >= 2^-900).  Operands
// outside these ranges (negative or non-finite) take the division.
CD_DEV bool depth_normal_ok(float Z, float Zp, float fwZ, float3 n, float3 np, float fwN)
{
    const float a = fabsf(__fsub_rn(Zp, Z)), b = __fadd_rn(fwZ, 1e-2f);
    const bool depth_bad = (b >= 0x1p-100f && b <= 0x1p100f && a <= 0x1p100f)
                               ? __fmaf_rn(-10.f, b, a) > __fmul_rn(b, 0x1p-21f)   // ulp(10) / 2 = 2^-21
                               : __fdiv_rn(a, b) > 10.f;
    if (depth_bad) return false;
    const float dx = __fsub_rn(n.x, np.x), dy = __fsub_rn(n.y, np.y), dz = __fsub_rn(n.z, np.z);
    const float dd = __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
    const float dist = __fsqrt_rn(dd);
    const double S = __dadd_rn((double)fwN, 1e-2);
    const bool normal_bad = (S >= 0x1p-900 && S <= 0x1p900 && dist <= 0x1p100f)
                                ? __fma_rn(-4.0, S, (double)dist) > __dmul_rn(S, 0x1p-51)   // ulp(4) / 2 = 2^-51
                                : __ddiv_rn((double)dist, S) > 4.0;
    return !normal_bad;
}

template <int kN, int kC>
__global__ void __launch_bounds__(256) reproject_kernel(
    const float *__restrict__ mvec, ReprojectList list, const float *__restrict__ linz,
    const float *__restrict__ plinz, const float *__restrict__ nrm,
    const float *__restrict__ pnrm, const float *__restrict__ pnfw,
    const float *__restrict__ opac, const float *__restrict__ popac,
    uint8_t *__restrict__ success, int H, int W)
{
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    const int cy = blockIdx.y * blockDim.y + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const size_t base = (size_t)blockIdx.z * H * W;
    const size_t c = base + (size_t)cy * W + cx;
    const int n_list = kN > 0 ? kN : list.n;

    // tap selection: mode 0 = none, 1 = bilinear (weights w[], divide by
    // sumw), 2 = 3x3 box (bitmask box, divide by the count)
    int mode = 0;
    float w[4] = {0.f, 0.f, 0.f, 0.f};
    float norm = 1.f;
    unsigned vmask = 0u, box = 0u;
    int lx = 0, ly = 0, ipx = 0, ipy = 0;

    // own-pixel inputs loaded together, not behind the opacity test
    const float op = __ldg(opac + c), mx = __ldg(mvec + 3 * c), my = __ldg(mvec + 3 * c + 1);
    const float fwN = __ldg(pnfw + 3 * c + 1);
    const float Z = __ldg(linz + 3 * c), fwZ = __ldg(linz + 3 * c + 1);
    const float3 n = ld3(nrm, c);
    if (op != 0.f) {
        const float fW = (float)W, fH = (float)H, fx = (float)cx, fy = (float)cy;
        // iposPrev = int(pos + mvec * dim + 0.5)   (line 97)
        ipx = __float2int_rz(__fadd_rn(__fmaf_rn(mx, fW, fx), 0.5f));
        ipy = __float2int_rz(__fadd_rn(__fmaf_rn(my, fH, fy), 0.5f));
        // posPrev = floor(pos) + mvec * dim       (line 103)
        const float ppx = __fmaf_rn(mx, fW, floorf(fx));
        const float ppy = __fmaf_rn(my, fH, floorf(fy));
        lx = __float2int_rz(ppx);
        ly = __float2int_rz(ppy);
        const bool border_ok = !(ipx < 1 || ipy < 1 || ipx > W - 1 || ipy > H - 1);

        if (border_ok) {
            // the four taps' previous opacity, depth and normal, all loads
            // issued before the first test
            float po[4], zp[4];
            float3 np[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int qx = lx + (s & 1), qy = ly + (s >> 1);
                po[s] = 0.f;
                if (qx >= W || qx < 0 || qy >= H || qy < 0) continue;
                const size_t q = base + (size_t)qy * W + qx;
                po[s] = __ldg(popac + q);
                zp[s] = __ldg(plinz + 3 * q);
                np[s] = ld3(pnrm, q);
            }
#pragma unroll
            for (int s = 0; s < 4; ++s)
                if (po[s] != 0.f && depth_normal_ok(Z, zp[s], fwZ, n, np[s], fwN)) vmask |= 1u << s;
        }
        if (vmask) {
            // bilinear weights from the fractional part (line 130-137)
            const float x = __fsub_rn(ppx, floorf(ppx)), y = __fsub_rn(ppy, floorf(ppy));
            const float a0 = __fsub_rn(1.f, x), b0 = __fsub_rn(1.f, y);
            const float fa[4] = {a0, x, a0, x}, fb[4] = {b0, b0, y, y};
            float sumw = 0.f;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                w[s] = __fmul_rn(fa[s], fb[s]);
                // the weight sum adds the rounded weights (no fused multiply-add)
                if (vmask & (1u << s)) sumw = __fadd_rn(sumw, w[s]);
            }
            if (sumw >= 0.01f) {
                mode = 1;
                norm = sumw;
            }
        }
        if (mode == 0 && border_ok) {
            int cnt = 0;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int qx = ipx + (k % 3) - 1, qy = ipy + (k / 3) - 1;
                if (qx >= W || qx < 0 || qy >= H || qy < 0) continue;
                // the reference reads prev_opacity here without the batch
                // offset (ops/reproject.cu.cc:191)
                if (__ldg(popac + (size_t)qy * W + qx) == 0.f) continue;
                const size_t q = base + (size_t)qy * W + qx;
                if (depth_normal_ok(Z, __ldg(plinz + 3 * q), fwZ, n, ld3(pnrm, q), fwN)) {
                    box |= 1u << k;
                    ++cnt;
                }
            }
            if (cnt > 0) {
                mode = 2;
                norm = (float)cnt;
            }
        }
    }
    success[c] = mode != 0;

    // gather and write every output value once
    for (int d = 0; d < n_list; ++d) {
        const int C = kC > 0 ? kC : list.ch[d];
        const float *in = list.in[d];
        float *out = list.out[d] + c * C;
        for (int k = 0; k < C; ++k) {
            float acc = 0.f;
            if (mode == 1) {
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    if (vmask & (1u << s)) {
                        const size_t q = base + (size_t)(ly + (s >> 1)) * W + (lx + (s & 1));
                        acc = __fmaf_rn(w[s], __ldg(in + q * C + k), acc);
                    }
                acc = __fdiv_rn(acc, norm);
            } else if (mode == 2) {
#pragma unroll
                for (int s = 0; s < 9; ++s)
                    if (box & (1u << s)) {
                        const size_t q = base + (size_t)(ipy + s / 3 - 1) * W + (ipx + s % 3 - 1);
                        acc = __fadd_rn(acc, __ldg(in + q * C + k));
                    }
                acc = __fdiv_rn(acc, norm);
            }
            out[k] = acc;
        }
    }
}

// Two-kernel form of the 3-tensor, 3-channel list (the per-frame step's):
// the same decisions and arithmetic as reproject_kernel<3, 3>, split so that
// each kernel has two dependent load rounds and few live registers.
// reproject_decide_kernel reads the pixel's own inputs and its taps and
// leaves its decision in the success byte: 0 none, 0x10 | vmask bilinear
// (bit s = tap s valid), 0x20 the 3x3 box.  reproject_gather_kernel
// re-derives the taps and weights from the motion vector, re-tests the box
// (its rare case), gathers the history tensors, writes every output once
// and the final success byte.
constexpr uint8_t kModeBilinear = 0x10, kModeBox = 0x20;

CD_DEV void reproject_taps(float mx, float my, int cx, int cy, int W, int H, int &ipx, int &ipy, float &ppx,
                           float &ppy)
{
    const float fW = (float)W, fH = (float)H, fx = (float)cx, fy = (float)cy;
    ipx = __float2int_rz(__fadd_rn(__fmaf_rn(mx, fW, fx), 0.5f));
    ipy = __float2int_rz(__fadd_rn(__fmaf_rn(my, fH, fy), 0.5f));
    ppx = __fmaf_rn(mx, fW, floorf(fx));
    ppy = __fmaf_rn(my, fH, floorf(fy));
}

// bilinear weights of the four taps and their sum over vmask
CD_DEV float bilinear(float ppx, float ppy, unsigned vmask, float w[4])
{
    const float x = __fsub_rn(ppx, floorf(ppx)), y = __fsub_rn(ppy, floorf(ppy));
    const float a0 = __fsub_rn(1.f, x), b0 = __fsub_rn(1.f, y);
    const float fa[4] = {a0, x, a0, x}, fb[4] = {b0, b0, y, y};
    float sumw = 0.f;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        w[s] = __fmul_rn(fa[s], fb[s]);
        if (vmask & (1u << s)) sumw = __fadd_rn(sumw, w[s]);
    }
    return sumw;
}

__global__ void __launch_bounds__(256) reproject_decide_kernel(
    const float *__restrict__ mvec, const float *__restrict__ linz, const float *__restrict__ plinz,
    const float *__restrict__ nrm, const float *__restrict__ pnrm, const float *__restrict__ pnfw,
    const float *__restrict__ opac, const float *__restrict__ popac, uint8_t *__restrict__ success, int H, int W)
{
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    const int cy = blockIdx.y * blockDim.y + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const size_t base = (size_t)blockIdx.z * H * W;
    const size_t c = base + (size_t)cy * W + cx;
    uint8_t code = 0;
    const float op = __ldg(opac + c), mx = __ldg(mvec + 3 * c), my = __ldg(mvec + 3 * c + 1);
    const float fwN = __ldg(pnfw + 3 * c + 1);
    const float Z = __ldg(linz + 3 * c), fwZ = __ldg(linz + 3 * c + 1);
    const float3 n = ld3(nrm, c);
    if (op != 0.f) {
        int ipx, ipy;
        float ppx, ppy;
        reproject_taps(mx, my, cx, cy, W, H, ipx, ipy, ppx, ppy);
        const int lx = __float2int_rz(ppx), ly = __float2int_rz(ppy);
        const bool border_ok = !(ipx < 1 || ipy < 1 || ipx > W - 1 || ipy > H - 1);
        unsigned vmask = 0u;
        if (border_ok) {
            float po[4], zp[4];
            float3 np[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int qx = lx + (s & 1), qy = ly + (s >> 1);
                po[s] = 0.f;
                if (qx >= W || qx < 0 || qy >= H || qy < 0) continue;
                const size_t q = base + (size_t)qy * W + qx;
                po[s] = __ldg(popac + q);
                zp[s] = __ldg(plinz + 3 * q);
                np[s] = ld3(pnrm, q);
            }
#pragma unroll
            for (int s = 0; s < 4; ++s)
                if (po[s] != 0.f && depth_normal_ok(Z, zp[s], fwZ, n, np[s], fwN)) vmask |= 1u << s;
        }
        float w[4];
        if (vmask && bilinear(ppx, ppy, vmask, w) >= 0.01f) {
            code = (uint8_t)(kModeBilinear | vmask);
        } else if (border_ok) {
#pragma unroll
            for (int k = 0; k < 9 && code == 0; ++k) {
                const int qx = ipx + (k % 3) - 1, qy = ipy + (k / 3) - 1;
                if (qx >= W || qx < 0 || qy >= H || qy < 0) continue;
                // the reference reads prev_opacity here without the batch
                // offset (ops/reproject.cu.cc:191)
                if (__ldg(popac + (size_t)qy * W + qx) == 0.f) continue;
                const size_t q = base + (size_t)qy * W + qx;
                if (depth_normal_ok(Z, __ldg(plinz + 3 * q), fwZ, n, ld3(pnrm, q), fwN)) code = kModeBox;
            }
        }
    }
    success[c] = code;
}

__global__ void __launch_bounds__(256) reproject_gather_kernel(
    const float *__restrict__ mvec, ReprojectList list, const float *__restrict__ linz,
    const float *__restrict__ plinz, const float *__restrict__ nrm, const float *__restrict__ pnrm,
    const float *__restrict__ pnfw, const float *__restrict__ popac, uint8_t *__restrict__ success, int H, int W)
{
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    const int cy = blockIdx.y * blockDim.y + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const size_t base = (size_t)blockIdx.z * H * W;
    const size_t c = base + (size_t)cy * W + cx;
    const uint8_t code = success[c];
    float acc[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d][0] = acc[d][1] = acc[d][2] = 0.f;
    float norm = 1.f;
    if (code) {
        const float mx = __ldg(mvec + 3 * c), my = __ldg(mvec + 3 * c + 1);
        int ipx, ipy;
        float ppx, ppy;
        reproject_taps(mx, my, cx, cy, W, H, ipx, ipy, ppx, ppy);
        if (code & kModeBilinear) {
            const unsigned vmask = code & 0xFu;
            float w[4];
            norm = bilinear(ppx, ppy, vmask, w);
            const int lx = __float2int_rz(ppx), ly = __float2int_rz(ppy);
            float3 g[3][4];
#pragma unroll
            for (int s = 0; s < 4; ++s)
                if (vmask & (1u << s)) {
                    const size_t q = base + (size_t)(ly + (s >> 1)) * W + (lx + (s & 1));
#pragma unroll
                    for (int d = 0; d < 3; ++d) g[d][s] = ld3(list.in[d], q);
                }
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    if (vmask & (1u << s)) {
                        acc[d][0] = __fmaf_rn(w[s], g[d][s].x, acc[d][0]);
                        acc[d][1] = __fmaf_rn(w[s], g[d][s].y, acc[d][1]);
                        acc[d][2] = __fmaf_rn(w[s], g[d][s].z, acc[d][2]);
                    }
        } else {
            // the 3x3 box, re-tested (the decision kernel keeps one bit)
            const float fwN = __ldg(pnfw + 3 * c + 1);
            const float Z = __ldg(linz + 3 * c), fwZ = __ldg(linz + 3 * c + 1);
            const float3 n = ld3(nrm, c);
            int cnt = 0;
            for (int k = 0; k < 9; ++k) {
                const int qx = ipx + (k % 3) - 1, qy = ipy + (k / 3) - 1;
                if (qx >= W || qx < 0 || qy >= H || qy < 0) continue;
                if (__ldg(popac + (size_t)qy * W + qx) == 0.f) continue;
                const size_t q = base + (size_t)qy * W + qx;
                if (!depth_normal_ok(Z, __ldg(plinz + 3 * q), fwZ, n, ld3(pnrm, q), fwN)) continue;
                ++cnt;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const float3 v = ld3(list.in[d], q);
                    acc[d][0] = __fadd_rn(acc[d][0], v.x);
                    acc[d][1] = __fadd_rn(acc[d][1], v.y);
                    acc[d][2] = __fadd_rn(acc[d][2], v.z);
                }
            }
            norm = (float)cnt;
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float *out = list.out[d] + c * 3;
#pragma unroll
        for (int k = 0; k < 3; ++k) out[k] = code ? __fdiv_rn(acc[d][k], norm) : 0.f;
    }
    success[c] = code != 0;
}

}  // namespace

cudaError_t launch_reproject(const float *mvec, const ReprojectList &list, const float *linz,
                             const float *plinz, const float *nrm, const float *pnrm,
                             const float *pnfw, const float *opac, const float *popac,
                             uint8_t *success, int B, int H, int W, cudaStream_t st)
{
    dim3 block(32, 8);
    dim3 grid((W + 31) / 32, (H + 7) / 8, B);
    bool fast = list.n == 3;
    for (int d = 0; d < list.n; ++d) fast = fast && list.ch[d] == 3;
    if (fast) {
        reproject_decide_kernel<<<grid, block, 0, st>>>(mvec, linz, plinz, nrm, pnrm, pnfw, opac, popac, success,
                                                        H, W);
        reproject_gather_kernel<<<grid, block, 0, st>>>(mvec, list, linz, plinz, nrm, pnrm, pnfw, popac, success, H,
                                                        W);
    }
    else
        reproject_kernel<0, 0><<<grid, block, 0, st>>>(mvec, list, linz, plinz, nrm, pnrm, pnfw,
                                                       opac, popac, success, H, W);
    return cudaGetLastError();
}

}  // namespace cd
