// Cross-regression on sm_100a: variance estimate, per-centre weighted least
// squares and block reconstruction.
//
// Reference semantics: ops/regression.cu.cc:206-500 (EstInputVarianceKernel,
// RegressionKernel with cholesky_color / forward_backward_solver, BlockRecon,
// CrossRegressionFunc).  Buffer A regresses imgb (target) on imga's features
// and buffer B the converse; both are computed by the same threads so the
// albedo / normal differences and the shared tile are read once.
//
// Coefficient layout in the workspace: beta[buf][b][j][i][r][ch] with
// r = 0..5 the regression coefficient (constant, colour, albedo, normal.xyz)
// and ch = 0..2 the colour channel; 18 floats per centre and buffer.
#include <cuda_runtime.h>
#include "cd_common.cuh"

namespace cd {
namespace {

constexpr int kP = 6;            // coefficients per channel (ops/regression.cu.cc:30)
constexpr int kBeta = kP * 3;    // floats per centre and buffer

// ---------------------------------------------------------------------------
// Variance: var = |mean of the in-bounds 3x3 neighbours minus the centre -
// centre|^2 summed over channels (ops/regression.cu.cc:244-276).
// blockIdx.z = 2 * batch + buffer.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) variance_kernel(const float *__restrict__ imga,
                                                       const float *__restrict__ imgb,
                                                       float *__restrict__ vara,
                                                       float *__restrict__ varb, int H, int W)
{
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    const int cy = blockIdx.y * blockDim.y + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const int buf = blockIdx.z & 1;
    const size_t base = (size_t)(blockIdx.z >> 1) * H * W;
    const float *img = (buf ? imgb : imga) + 3 * base;
    float *var = (buf ? varb : vara) + base;
    const int sx = max(0, cx - 1), ex = min(W - 1, cx + 1);
    const int sy = max(0, cy - 1), ey = min(H - 1, cy + 1);
    float ax = 0.f, ay = 0.f, az = 0.f;
    int n = 0;
    for (int iy = sy; iy <= ey; ++iy)
        for (int ix = sx; ix <= ex; ++ix) {
            if (iy == cy && ix == cx) continue;
            const float3 v = ld3(img, (size_t)iy * W + ix);
            ax += v.x;
            ay += v.y;
            az += v.z;
            ++n;
        }
    const float fn = (float)n;
    const float3 c = ld3(img, (size_t)cy * W + cx);
    var[(size_t)cy * W + cx] = norm2(ax / fn - c.x, ay / fn - c.y, az / fn - c.z);
}

// ---------------------------------------------------------------------------
// Normal-equation accumulators of one buffer.  The 6x6 per-channel systems
// share every entry that involves only the constant and the normal
// differences, so 61 scalars describe all three channels:
//   shared (10): A00 A03 A04 A05 A33 A34 A35 A44 A45 A55
//   per channel (11 x 3): A01 A02 A11 A12 A13 A14 A15 A22 A23 A24 A25
//   right-hand side (6 x 3): X0..X5
// ---------------------------------------------------------------------------
struct Normal {
    float a00, a03, a04, a05, a33, a34, a35, a44, a45, a55;
    float a01[3], a02[3], a11[3], a12[3], a13[3], a14[3], a15[3], a22[3], a23[3], a24[3], a25[3];
    float x0[3], x1[3], x2[3], x3[3], x4[3], x5[3];
};

CD_DEV void normal_zero(Normal &n)
{
    n.a00 = n.a03 = n.a04 = n.a05 = n.a33 = n.a34 = n.a35 = n.a44 = n.a45 = n.a55 = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        n.a01[k] = n.a02[k] = n.a11[k] = n.a12[k] = n.a13[k] = n.a14[k] = n.a15[k] = 0.f;
        n.a22[k] = n.a23[k] = n.a24[k] = n.a25[k] = 0.f;
        n.x0[k] = n.x1[k] = n.x2[k] = n.x3[k] = n.x4[k] = n.x5[k] = 0.f;
    }
}

// One window tap of one buffer: features f (centre fc), target y, variance
// and standard deviation (v, sd), shared albedo / normal differences.
// Follows ops/regression.cu.cc:418-445: delta = [1, (f_t-f_c)/(sd_c+sd_t+1e-2),
// alb_t-alb_c, n_t-n_c], w = exp(-|f_t-f_c|^2/(v_c+v_t+1e-4)) + 1e-7.
CD_DEV void normal_tap(Normal &n, float3 ft, float3 fc, float3 y, float vt, float vc, float sdt,
                       float sdc, const float da[3], const float dn[3])
{
    const float df[3] = {ft.x - fc.x, ft.y - fc.y, ft.z - fc.z};
    const float den = (sdc + sdt) + 1e-2f;
    const float dist = norm2(df[0], df[1], df[2]) / ((vc + vt) + 1e-4f);
    const float w = __expf(-dist) + 1e-7f;
    const float wn0 = w * dn[0], wn1 = w * dn[1], wn2 = w * dn[2];
    n.a00 += w;
    n.a03 = fmaf(w, dn[0], n.a03);
    n.a04 = fmaf(w, dn[1], n.a04);
    n.a05 = fmaf(w, dn[2], n.a05);
    n.a33 = fmaf(wn0, dn[0], n.a33);
    n.a34 = fmaf(wn0, dn[1], n.a34);
    n.a35 = fmaf(wn0, dn[2], n.a35);
    n.a44 = fmaf(wn1, dn[1], n.a44);
    n.a45 = fmaf(wn1, dn[2], n.a45);
    n.a55 = fmaf(wn2, dn[2], n.a55);
    const float yv[3] = {y.x, y.y, y.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float d1 = df[k] / den;
        const float wd1 = w * d1, wd2 = w * da[k];
        n.a01[k] = fmaf(w, d1, n.a01[k]);
        n.a02[k] = fmaf(w, da[k], n.a02[k]);
        n.a11[k] = fmaf(wd1, d1, n.a11[k]);
        n.a12[k] = fmaf(wd1, da[k], n.a12[k]);
        n.a13[k] = fmaf(wd1, dn[0], n.a13[k]);
        n.a14[k] = fmaf(wd1, dn[1], n.a14[k]);
        n.a15[k] = fmaf(wd1, dn[2], n.a15[k]);
        n.a22[k] = fmaf(wd2, da[k], n.a22[k]);
        n.a23[k] = fmaf(wd2, dn[0], n.a23[k]);
        n.a24[k] = fmaf(wd2, dn[1], n.a24[k]);
        n.a25[k] = fmaf(wd2, dn[2], n.a25[k]);
        n.x0[k] = fmaf(w, yv[k], n.x0[k]);
        n.x1[k] = fmaf(wd1, yv[k], n.x1[k]);
        n.x2[k] = fmaf(wd2, yv[k], n.x2[k]);
        n.x3[k] = fmaf(wn0, yv[k], n.x3[k]);
        n.x4[k] = fmaf(wn1, yv[k], n.x4[k]);
        n.x5[k] = fmaf(wn2, yv[k], n.x5[k]);
    }
}

// Sum the accumulators over the `width` lanes of a group (xor butterfly, so
// every lane of the group ends with the same total).
CD_DEV float group_sum(float v, int width)
{
    for (int m = 1; m < width; m <<= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;
}

CD_DEV void normal_reduce(Normal &n, int width)
{
    if (width == 1) return;
    n.a00 = group_sum(n.a00, width);
    n.a03 = group_sum(n.a03, width);
    n.a04 = group_sum(n.a04, width);
    n.a05 = group_sum(n.a05, width);
    n.a33 = group_sum(n.a33, width);
    n.a34 = group_sum(n.a34, width);
    n.a35 = group_sum(n.a35, width);
    n.a44 = group_sum(n.a44, width);
    n.a45 = group_sum(n.a45, width);
    n.a55 = group_sum(n.a55, width);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        n.a01[k] = group_sum(n.a01[k], width);
        n.a02[k] = group_sum(n.a02[k], width);
        n.a11[k] = group_sum(n.a11[k], width);
        n.a12[k] = group_sum(n.a12[k], width);
        n.a13[k] = group_sum(n.a13[k], width);
        n.a14[k] = group_sum(n.a14[k], width);
        n.a15[k] = group_sum(n.a15[k], width);
        n.a22[k] = group_sum(n.a22[k], width);
        n.a23[k] = group_sum(n.a23[k], width);
        n.a24[k] = group_sum(n.a24[k], width);
        n.a25[k] = group_sum(n.a25[k], width);
        n.x0[k] = group_sum(n.x0[k], width);
        n.x1[k] = group_sum(n.x1[k], width);
        n.x2[k] = group_sum(n.x2[k], width);
        n.x3[k] = group_sum(n.x3[k], width);
        n.x4[k] = group_sum(n.x4[k], width);
        n.x5[k] = group_sum(n.x5[k], width);
    }
}

// Cholesky factorisation + forward / backward substitution of one channel's
// ridge-regularised 6x6 system, in the reference's operation order
// (ops/regression.cu.cc:206-242, 449-467): diagonal pivots
// sqrt(max(1e-5, a_ii - s)), off-diagonals (1/L_jj) * (a_ji - s).
CD_DEV void solve_channel(const Normal &n, int k, float *beta)
{
    float A[kP][kP];
    A[0][0] = n.a00; A[0][1] = n.a01[k]; A[0][2] = n.a02[k]; A[0][3] = n.a03; A[0][4] = n.a04; A[0][5] = n.a05;
    A[1][1] = n.a11[k]; A[1][2] = n.a12[k]; A[1][3] = n.a13[k]; A[1][4] = n.a14[k]; A[1][5] = n.a15[k];
    A[2][2] = n.a22[k]; A[2][3] = n.a23[k]; A[2][4] = n.a24[k]; A[2][5] = n.a25[k];
    A[3][3] = n.a33; A[3][4] = n.a34; A[3][5] = n.a35;
    A[4][4] = n.a44; A[4][5] = n.a45;
    A[5][5] = n.a55;
#pragma unroll
    for (int r = 0; r < kP; ++r) A[r][r] += 1e-3f;
    const float X[kP] = {n.x0[k], n.x1[k], n.x2[k], n.x3[k], n.x4[k], n.x5[k]};
    float L[kP][kP];
#pragma unroll
    for (int i = 0; i < kP; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            float s = 0.f;
#pragma unroll
            for (int q = 0; q < j; ++q) s = fmaf(L[i][q], L[j][q], s);
            if (i == j)
                L[i][i] = sqrtf(fmaxf(1e-5f, A[i][i] - s));
            else
                L[i][j] = (1.f / L[j][j]) * (A[j][i] - s);
        }
    }
    float Y[kP];
    Y[0] = X[0] / L[0][0];
#pragma unroll
    for (int i = 1; i < kP; ++i) {
        float s = 0.f;
#pragma unroll
        for (int q = 0; q < i; ++q) s = fmaf(L[i][q], Y[q], s);
        Y[i] = (X[i] - s) / L[i][i];
    }
    float bt[kP];
    bt[kP - 1] = Y[kP - 1] / L[kP - 1][kP - 1];
#pragma unroll
    for (int i = kP - 2; i >= 0; --i) {
        float s = 0.f;
#pragma unroll
        for (int q = kP - 1; q > i; --q) s = fmaf(L[q][i], bt[q], s);
        bt[i] = (Y[i] - s) / L[i][i];
    }
#pragma unroll
    for (int r = 0; r < kP; ++r) beta[r * 3 + k] = bt[r];
}

// ---------------------------------------------------------------------------
// Regression kernel.
// A CTA owns a tile of kTCX x kTCY centres.  Its window footprint (centres
// plus the window radius on every side, reflect-101 at the image border) is
// staged once in shared memory as 16 SoA planes: imga.xyz, imgb.xyz,
// albedo.xyz, normal.xyz, varA, varB, sdA, sdB.  Four lanes work on one
// centre and split the window rows (lane j takes rows j, j+4, ...); each lane
// accumulates both buffers' normal equations in registers, the four partial
// sums are combined with warp shuffles, and the six channel systems
// (3 channels x 2 buffers) are solved by the four lanes in registers.
// With centres 4 px apart and an odd plane pitch the 32 lanes of a warp read
// 32 distinct banks.
// ---------------------------------------------------------------------------
constexpr int kTCX = 8;       // centres per CTA along x (one warp row)
constexpr int kLanes = 4;     // lanes per centre
constexpr int kPlanes = 16;

struct TileGeom {
    int tcy;        // centres per CTA along y (= warps per CTA)
    int pw, ph;     // footprint in pixels
    int pitch;      // plane row pitch (odd)
    size_t smem;    // bytes
};

__host__ __device__ inline TileGeom tile_geom(int hw, int sp, int tcy)
{
    TileGeom g;
    g.tcy = tcy;
    g.pw = (kTCX - 1) * sp + 2 * hw + 1;
    g.ph = (tcy - 1) * sp + 2 * hw + 1;
    g.pitch = g.pw | 1;
    g.smem = (size_t)kPlanes * g.ph * g.pitch * sizeof(float);
    return g;
}

__global__ void __launch_bounds__(256) regression_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ vara, const float *__restrict__ varb, float *__restrict__ beta,
    int H, int W, int hw, int sp, int tcy)
{
    extern __shared__ float smem[];
    const TileGeom g = tile_geom(hw, sp, tcy);
    const int plane = g.ph * g.pitch;
    const int Ws = W / sp, Hs = H / sp;
    const int b = blockIdx.z;
    const size_t px = (size_t)H * W;
    imga += 3 * px * b;
    imgb += 3 * px * b;
    albedo += 3 * px * b;
    normal += 3 * px * b;
    vara += px * b;
    varb += px * b;

    const int i0 = blockIdx.x * kTCX, j0 = blockIdx.y * tcy;
    const int x0 = i0 * sp - hw, y0 = j0 * sp - hw;

    // Stage the footprint.  Pixels past the reflect range belong to no valid
    // centre's window; they are clamped only to keep the loads in bounds.
    for (int t = threadIdx.x; t < g.pw * g.ph; t += blockDim.x) {
        const int ty = t / g.pw, tx = t - ty * g.pw;
        const int gx = min(max(mirror(x0 + tx, W), 0), W - 1);
        const int gy = min(max(mirror(y0 + ty, H), 0), H - 1);
        const size_t q = (size_t)gy * W + gx;
        const int o = ty * g.pitch + tx;
        const float3 a = ld3(imga, q), bb = ld3(imgb, q), al = ld3(albedo, q), nr = ld3(normal, q);
        const float va = __ldg(vara + q), vb = __ldg(varb + q);
        smem[0 * plane + o] = a.x;
        smem[1 * plane + o] = a.y;
        smem[2 * plane + o] = a.z;
        smem[3 * plane + o] = bb.x;
        smem[4 * plane + o] = bb.y;
        smem[5 * plane + o] = bb.z;
        smem[6 * plane + o] = al.x;
        smem[7 * plane + o] = al.y;
        smem[8 * plane + o] = al.z;
        smem[9 * plane + o] = nr.x;
        smem[10 * plane + o] = nr.y;
        smem[11 * plane + o] = nr.z;
        smem[12 * plane + o] = va;
        smem[13 * plane + o] = vb;
        smem[14 * plane + o] = sqrtf(va);
        smem[15 * plane + o] = sqrtf(vb);
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int ci = lane / kLanes;          // centre column inside the tile
    const int sub = lane % kLanes;         // row slice of the window
    const int cj = threadIdx.x >> 5;       // centre row inside the tile (warp)
    const int ctx = ci * sp + hw, cty = cj * sp + hw;   // centre in tile coordinates
    const int co = cty * g.pitch + ctx;

    const float3 fa_c = make_float3(smem[co], smem[plane + co], smem[2 * plane + co]);
    const float3 fb_c = make_float3(smem[3 * plane + co], smem[4 * plane + co], smem[5 * plane + co]);
    const float al_c[3] = {smem[6 * plane + co], smem[7 * plane + co], smem[8 * plane + co]};
    const float nr_c[3] = {smem[9 * plane + co], smem[10 * plane + co], smem[11 * plane + co]};
    const float va_c = smem[12 * plane + co], vb_c = smem[13 * plane + co];
    const float sa_c = smem[14 * plane + co], sb_c = smem[15 * plane + co];

    Normal na, nb;
    normal_zero(na);
    normal_zero(nb);

    for (int dy = -hw + sub; dy <= hw; dy += kLanes) {
        const int rowo = (cty + dy) * g.pitch + ctx;
        for (int dx = -hw; dx <= hw; ++dx) {
            const int o = rowo + dx;
            const float3 ta = make_float3(smem[o], smem[plane + o], smem[2 * plane + o]);
            const float3 tb = make_float3(smem[3 * plane + o], smem[4 * plane + o], smem[5 * plane + o]);
            const float da[3] = {smem[6 * plane + o] - al_c[0], smem[7 * plane + o] - al_c[1],
                                 smem[8 * plane + o] - al_c[2]};
            const float dn[3] = {smem[9 * plane + o] - nr_c[0], smem[10 * plane + o] - nr_c[1],
                                 smem[11 * plane + o] - nr_c[2]};
            const float va_t = smem[12 * plane + o], vb_t = smem[13 * plane + o];
            const float sa_t = smem[14 * plane + o], sb_t = smem[15 * plane + o];
            normal_tap(na, ta, fa_c, tb, va_t, va_c, sa_t, sa_c, da, dn);
            normal_tap(nb, tb, fb_c, ta, vb_t, vb_c, sb_t, sb_c, da, dn);
        }
    }

    normal_reduce(na, kLanes);
    normal_reduce(nb, kLanes);

    const int ci_g = i0 + ci, cj_g = j0 + cj;
    if (ci_g >= Ws || cj_g >= Hs) return;
    const size_t nb_img = (size_t)Hs * Ws;
    const size_t cidx = (size_t)b * nb_img + (size_t)cj_g * Ws + ci_g;
    const size_t buf_stride = (size_t)gridDim.z * nb_img * kBeta;
    float *ba = beta + cidx * kBeta;
    float *bbp = beta + buf_stride + cidx * kBeta;
    // six (buffer, channel) systems over four lanes: lane s takes s and s+4
#pragma unroll
    for (int p = 0; p < 6; ++p) {
        if (p % kLanes != sub) continue;
        if (p < 3)
            solve_channel(na, p, ba);
        else
            solve_channel(nb, p - 3, bbp);
    }
}

// ---------------------------------------------------------------------------
// Block reconstruction (ops/regression.cu.cc:289-365).  Each thread owns one
// output pixel of both buffers and sums, over the centres inside its window
// (centre range clamped to the image with the reference's iDivUp), the
// weighted predictions beta_c . delta(p, c) with delta taken as (p - c).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) recon_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ vara, const float *__restrict__ varb,
    const float *__restrict__ beta, float *__restrict__ outa, float *__restrict__ outb,
    int H, int W, int hw, int sp, int rs)
{
    const int Wr = W / rs, Hr = H / rs;
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    const int cy = blockIdx.y * blockDim.y + threadIdx.y;
    if (cx >= Wr || cy >= Hr) return;
    const int b = blockIdx.z;
    const size_t px = (size_t)H * W;
    imga += 3 * px * b;
    imgb += 3 * px * b;
    albedo += 3 * px * b;
    normal += 3 * px * b;
    vara += px * b;
    varb += px * b;
    const int Ws = W / sp, Hs = H / sp;
    const size_t nb_img = (size_t)Hs * Ws;
    const float *betaA = beta + (size_t)b * nb_img * kBeta;
    const float *betaB = beta + (size_t)gridDim.z * nb_img * kBeta + (size_t)b * nb_img * kBeta;

    const int pxo = cx * rs, pyo = cy * rs;
    const size_t p = (size_t)pyo * W + pxo;
    const int sx = max(0, idivup(pxo - hw, sp));
    const int ex = min((W - 1) / sp, (pxo + hw) / sp);
    const int sy = max(0, idivup(pyo - hw, sp));
    const int ey = min((H - 1) / sp, (pyo + hw) / sp);

    const float3 fa = ld3(imga, p), fb = ld3(imgb, p), al = ld3(albedo, p), nr = ld3(normal, p);
    const float va = __ldg(vara + p), vb = __ldg(varb + p);
    const float sa = sqrtf(va), sb = sqrtf(vb);
    float oa[3] = {0.f, 0.f, 0.f}, ob[3] = {0.f, 0.f, 0.f};
    float swa = 0.f, swb = 0.f;
    for (int iy = sy; iy <= ey; ++iy) {
        for (int ix = sx; ix <= ex; ++ix) {
            const size_t t = (size_t)(iy * sp) * W + ix * sp;
            const size_t cb = ((size_t)iy * Ws + ix) * kBeta;
            const float3 ta = ld3(imga, t), tb = ld3(imgb, t), tal = ld3(albedo, t), tnr = ld3(normal, t);
            const float vta = __ldg(vara + t), vtb = __ldg(varb + t);
            const float da[3] = {al.x - tal.x, al.y - tal.y, al.z - tal.z};
            const float dn[3] = {nr.x - tnr.x, nr.y - tnr.y, nr.z - tnr.z};
            {
                const float df[3] = {fa.x - ta.x, fa.y - ta.y, fa.z - ta.z};
                const float den = (sa + sqrtf(vta)) + 1e-2f;
                const float dist = norm2(-df[0], -df[1], -df[2]) / ((va + vta) + 1e-4f);
                const float w = __expf(-dist) + 1e-7f;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float *bc = betaA + cb + k;
                    float pr = __ldg(bc);
                    pr = fmaf(__ldg(bc + 3), df[k] / den, pr);
                    pr = fmaf(__ldg(bc + 6), da[k], pr);
                    pr = fmaf(__ldg(bc + 9), dn[0], pr);
                    pr = fmaf(__ldg(bc + 12), dn[1], pr);
                    pr = fmaf(__ldg(bc + 15), dn[2], pr);
                    oa[k] = fmaf(w, pr, oa[k]);
                }
                swa += w;
            }
            {
                const float df[3] = {fb.x - tb.x, fb.y - tb.y, fb.z - tb.z};
                const float den = (sb + sqrtf(vtb)) + 1e-2f;
                const float dist = norm2(-df[0], -df[1], -df[2]) / ((vb + vtb) + 1e-4f);
                const float w = __expf(-dist) + 1e-7f;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float *bc = betaB + cb + k;
                    float pr = __ldg(bc);
                    pr = fmaf(__ldg(bc + 3), df[k] / den, pr);
                    pr = fmaf(__ldg(bc + 6), da[k], pr);
                    pr = fmaf(__ldg(bc + 9), dn[0], pr);
                    pr = fmaf(__ldg(bc + 12), dn[1], pr);
                    pr = fmaf(__ldg(bc + 15), dn[2], pr);
                    ob[k] = fmaf(w, pr, ob[k]);
                }
                swb += w;
            }
        }
    }
    const float dA = fmaxf(swa, 1e-7f), dB = fmaxf(swb, 1e-7f);
    const size_t o = (size_t)b * Hr * Wr + (size_t)cy * Wr + cx;
    st3(outa, o, make_float3(fmaxf(0.f, oa[0] / dA), fmaxf(0.f, oa[1] / dA), fmaxf(0.f, oa[2] / dA)));
    st3(outb, o, make_float3(fmaxf(0.f, ob[0] / dB), fmaxf(0.f, ob[1] / dB), fmaxf(0.f, ob[2] / dB)));
}

}  // namespace

cudaError_t launch_variance(const float *imga, const float *imgb, float *vara, float *varb,
                            int B, int H, int W, cudaStream_t st)
{
    dim3 block(32, 8);
    dim3 grid((W + 31) / 32, (H + 7) / 8, 2 * B);
    variance_kernel<<<grid, block, 0, st>>>(imga, imgb, vara, varb, H, W);
    return cudaGetLastError();
}

cudaError_t launch_regression(const float *imga, const float *imgb, const float *albedo,
                              const float *normal, const float *vara, const float *varb,
                              float *beta, int B, int H, int W, int win, int sp, cudaStream_t st)
{
    const int hw = win / 2;
    int tcy = 4;
    while (tcy > 1 && tile_geom(hw, sp, tcy).smem > 200 * 1024) tcy >>= 1;
    const TileGeom g = tile_geom(hw, sp, tcy);
    if (g.smem > 220 * 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(regression_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem);
    if (e != cudaSuccess) return e;
    const int Ws = W / sp, Hs = H / sp;
    dim3 grid((Ws + kTCX - 1) / kTCX, (Hs + tcy - 1) / tcy, B);
    regression_kernel<<<grid, 32 * tcy, g.smem, st>>>(imga, imgb, albedo, normal, vara, varb,
                                                      beta, H, W, hw, sp, tcy);
    return cudaGetLastError();
}

cudaError_t launch_recon(const float *imga, const float *imgb, const float *albedo,
                         const float *normal, const float *vara, const float *varb,
                         const float *beta, float *outa, float *outb, int B, int H, int W,
                         int win, int sp, int rs, cudaStream_t st)
{
    const int Wr = W / rs, Hr = H / rs;
    dim3 block(32, 8);
    dim3 grid((Wr + 31) / 32, (Hr + 7) / 8, B);
    recon_kernel<<<grid, block, 0, st>>>(imga, imgb, albedo, normal, vara, varb, beta, outa, outb,
                                         H, W, win / 2, sp, rs);
    return cudaGetLastError();
}

}  // namespace cd
