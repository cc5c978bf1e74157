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
#include "f32x2.cuh"
#include "window_rows.cuh"

namespace cd {
namespace {

constexpr int kP = 6;            // coefficients per channel (ops/regression.cu.cc:30)
constexpr int kBeta = kP * 3;    // floats per centre and buffer

// ---------------------------------------------------------------------------
// Variance: var = |mean of the in-bounds 3x3 neighbours minus the centre -
// centre|^2 summed over channels (ops/regression.cu.cc:244-276).  Also
// writes sqrt(var) to a workspace plane: the regression and reconstruction
// read the standard deviation of every tap.
//
// variance_kernel: one thread per pixel computes both buffers from the
// block's footprint in shared memory (rows of 40 pixels from x0 - 4, as
// stored: 3 floats per pixel), each row copied by one warp with one float4
// per lane.  Needs W % 4 == 0 and 16-byte aligned images, so that every
// float4 lies wholly inside or wholly outside an image row.
// variance_px_kernel (any W): one thread per pixel and buffer, global loads.
// blockIdx.z = 2 * batch + buffer there.
// ---------------------------------------------------------------------------
constexpr int kVX = 32, kVY = 8;
constexpr int kVRow = 3 * (kVX + 8), kVTH = kVY + 2;   // footprint row: 40 pixels x 3 floats

__global__ void __launch_bounds__(kVX * kVY) variance_kernel(const float *__restrict__ imga,
                                                             const float *__restrict__ imgb,
                                                             float *__restrict__ vara,
                                                             float *__restrict__ varb,
                                                             float *__restrict__ sda,
                                                             float *__restrict__ sdb, int H, int W)
{
    __shared__ __align__(16) float tile[2][kVTH][kVRow];
    const int x0 = blockIdx.x * kVX, y0 = blockIdx.y * kVY, xa = x0 - 4;
    const size_t base = (size_t)blockIdx.z * H * W;
    const int lane = threadIdx.x, warp = threadIdx.y;
    constexpr int kRows = 2 * kVTH, kIt = (kRows + kVY - 1) / kVY;
    float4 v[kIt];
    // every load issued before the first store
#pragma unroll
    for (int k = 0; k < kIt; ++k) {
        const int rr = warp + k * kVY, buf = rr >= kVTH, ty = rr - buf * kVTH, gy = y0 - 1 + ty;
        const int f = 3 * xa + 4 * lane;   // float offset in the image row
        v[k] = make_float4(0.f, 0.f, 0.f, 0.f);   // outside the image: never read
        if (rr < kRows && 4 * lane < kVRow && gy >= 0 && gy < H && f >= 0 && f + 4 <= 3 * W)
            v[k] = __ldg(reinterpret_cast<const float4 *>((buf ? imgb : imga) + 3 * (base + (size_t)gy * W) + f));
    }
#pragma unroll
    for (int k = 0; k < kIt; ++k) {
        const int rr = warp + k * kVY, buf = rr >= kVTH, ty = rr - buf * kVTH;
        if (rr < kRows && 4 * lane < kVRow) *reinterpret_cast<float4 *>(&tile[buf][ty][4 * lane]) = v[k];
    }
    __syncthreads();
    const int cx = x0 + lane, cy = y0 + warp;
    if (cx >= W || cy >= H) return;
    const size_t p = base + (size_t)cy * W + cx;
#pragma unroll
    for (int buf = 0; buf < 2; ++buf) {
        float ax = 0.f, ay = 0.f, az = 0.f;
        int n = 0;
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (dy == 0 && dx == 0) continue;
                const int ix = cx + dx, iy = cy + dy;
                if (ix < 0 || ix >= W || iy < 0 || iy >= H) continue;
                const float *t = &tile[buf][warp + 1 + dy][3 * (lane + 4 + dx)];
                ax += t[0];
                ay += t[1];
                az += t[2];
                ++n;
            }
        const float *t = &tile[buf][warp + 1][3 * (lane + 4)];
        float mx, my, mz;
        if (n == 8) {
            // interior pixels: a quotient by 8 is the product by 1/8, exactly
            // (__fmul_rn: rounded on its own, never fused into the subtraction)
            mx = __fmul_rn(ax, 0.125f);
            my = __fmul_rn(ay, 0.125f);
            mz = __fmul_rn(az, 0.125f);
        } else {
            const float fn = (float)n;
            mx = ax / fn;
            my = ay / fn;
            mz = az / fn;
        }
        const float var = norm2(mx - t[0], my - t[1], mz - t[2]);
        (buf ? varb : vara)[p] = var;
        (buf ? sdb : sda)[p] = sqrtf(var);
    }
}

__global__ void __launch_bounds__(256) variance_px_kernel(const float *__restrict__ imga,
                                                       const float *__restrict__ imgb,
                                                       float *__restrict__ vara,
                                                       float *__restrict__ varb,
                                                       float *__restrict__ sda,
                                                       float *__restrict__ sdb, int H, int W)
{
    const int cx = blockIdx.x * blockDim.x + threadIdx.x;
    const int cy = blockIdx.y * blockDim.y + threadIdx.y;
    if (cx >= W || cy >= H) return;
    const int buf = blockIdx.z & 1;
    const size_t base = (size_t)(blockIdx.z >> 1) * H * W;
    const float *img = (buf ? imgb : imga) + 3 * base;
    float *var = (buf ? varb : vara) + base;
    float *sd = (buf ? sdb : sda) + base;
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
    const float3 c = ld3(img, (size_t)cy * W + cx);
    float mx, my, mz;
    if (n == 8) {
        // interior pixels: a quotient by 8 is the product by 1/8, exactly
        // (__fmul_rn: rounded on its own, never fused into the subtraction)
        mx = __fmul_rn(ax, 0.125f);
        my = __fmul_rn(ay, 0.125f);
        mz = __fmul_rn(az, 0.125f);
    } else {
        const float fn = (float)n;
        mx = ax / fn;
        my = ay / fn;
        mz = az / fn;
    }
    const float v = norm2(mx - c.x, my - c.y, mz - c.z);
    var[(size_t)cy * W + cx] = v;
    sd[(size_t)cy * W + cx] = sqrtf(v);
}

// ---------------------------------------------------------------------------
// Normal-equation accumulators of one buffer.  The 6x6 per-channel systems
// share every entry that involves only the constant and the normal
// differences, so 61 scalars describe all three channels:
//   shared (10): A00 A03 A04 A05 A33 A34 A35 A44 A45 A55
//   per channel (11 x 3): A01 A02 A11 A12 A13 A14 A15 A22 A23 A24 A25
//   right-hand side (6 x 3): X0..X5
// The per-channel terms of channels 0 and 1 are packed FP32x2 pairs (low
// lane channel 0) updated by one fma.rn.f32x2 each, channel 2 stays scalar:
// every lane is rounded as the scalar update, in the same order.
// ---------------------------------------------------------------------------
struct Normal {
    float a00, a03, a04, a05, a33, a34, a35, a44, a45, a55;
    x2::f2 p01, p02, p11, p12, p13, p14, p15, p22, p23, p24, p25;   // channels 0, 1
    x2::f2 px0, px1, px2, px3, px4, px5;
    float q01, q02, q11, q12, q13, q14, q15, q22, q23, q24, q25;      // channel 2
    float qx0, qx1, qx2, qx3, qx4, qx5;
};

CD_DEV void normal_zero(Normal &n)
{
    n.a00 = n.a03 = n.a04 = n.a05 = n.a33 = n.a34 = n.a35 = n.a44 = n.a45 = n.a55 = 0.f;
    const x2::f2 z = x2::pack(0.f, 0.f);
    n.p01 = n.p02 = n.p11 = n.p12 = n.p13 = n.p14 = n.p15 = n.p22 = n.p23 = n.p24 = n.p25 = z;
    n.px0 = n.px1 = n.px2 = n.px3 = n.px4 = n.px5 = z;
    n.q01 = n.q02 = n.q11 = n.q12 = n.q13 = n.q14 = n.q15 = n.q22 = n.q23 = n.q24 = n.q25 = 0.f;
    n.qx0 = n.qx1 = n.qx2 = n.qx3 = n.qx4 = n.qx5 = 0.f;
}

// channel k (0, 1: a lane of the pair; 2: the scalar) of a per-channel term
CD_DEV float chan(x2::f2 p, float q, int k) { return k == 0 ? x2::lo(p) : k == 1 ? x2::hi(p) : q; }

// |v|^2 as the reference's compiled norm2 rounds it: fma(z, z, fma(x, x, y*y))
// (the contraction the reference kernels were observed to use for
// x*x + y*y + z*z, see reproject.cu).
CD_DEV float sqnorm(float x, float y, float z) { return fmaf(z, z, fmaf(x, x, y * y)); }

// One window tap of one buffer: features f (centre fc), target y, variance
// and standard deviation (v, sd), shared albedo / normal differences.
// Follows ops/regression.cu.cc:418-445: delta = [1, (f_t-f_c)/(sd_c+sd_t+1e-2),
// alb_t-alb_c, n_t-n_c], w = exp(-|f_t-f_c|^2/(v_c+v_t+1e-4)) + 1e-7.
CD_DEV void normal_tap(Normal &n, float3 ft, float3 fc, float3 y, float vt, float vc, float sdt,
                       float sdc, const float da[3], const float dn[3])
{
    using namespace x2;
    const float df[3] = {ft.x - fc.x, ft.y - fc.y, ft.z - fc.z};
    const float den = (sdc + sdt) + 1e-2f;
    const float dist = sqnorm(df[0], df[1], df[2]) / ((vc + vt) + 1e-4f);
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
    // channels 0 and 1
    const f2 wP = pack(w, w), d1P = pack(df[0] / den, df[1] / den), daP = pack(da[0], da[1]);
    const f2 wd1P = mul2(wP, d1P), wd2P = mul2(wP, daP);
    const f2 dn0P = pack(dn[0], dn[0]), dn1P = pack(dn[1], dn[1]), dn2P = pack(dn[2], dn[2]);
    const f2 yP = pack(y.x, y.y);
    n.p01 = fma2(wP, d1P, n.p01);
    n.p02 = fma2(wP, daP, n.p02);
    n.p11 = fma2(wd1P, d1P, n.p11);
    n.p12 = fma2(wd1P, daP, n.p12);
    n.p13 = fma2(wd1P, dn0P, n.p13);
    n.p14 = fma2(wd1P, dn1P, n.p14);
    n.p15 = fma2(wd1P, dn2P, n.p15);
    n.p22 = fma2(wd2P, daP, n.p22);
    n.p23 = fma2(wd2P, dn0P, n.p23);
    n.p24 = fma2(wd2P, dn1P, n.p24);
    n.p25 = fma2(wd2P, dn2P, n.p25);
    n.px0 = fma2(wP, yP, n.px0);
    n.px1 = fma2(wd1P, yP, n.px1);
    n.px2 = fma2(wd2P, yP, n.px2);
    n.px3 = fma2(pack(wn0, wn0), yP, n.px3);
    n.px4 = fma2(pack(wn1, wn1), yP, n.px4);
    n.px5 = fma2(pack(wn2, wn2), yP, n.px5);
    // channel 2
    const float d1 = df[2] / den;
    const float wd1 = w * d1, wd2 = w * da[2];
    n.q01 = fmaf(w, d1, n.q01);
    n.q02 = fmaf(w, da[2], n.q02);
    n.q11 = fmaf(wd1, d1, n.q11);
    n.q12 = fmaf(wd1, da[2], n.q12);
    n.q13 = fmaf(wd1, dn[0], n.q13);
    n.q14 = fmaf(wd1, dn[1], n.q14);
    n.q15 = fmaf(wd1, dn[2], n.q15);
    n.q22 = fmaf(wd2, da[2], n.q22);
    n.q23 = fmaf(wd2, dn[0], n.q23);
    n.q24 = fmaf(wd2, dn[1], n.q24);
    n.q25 = fmaf(wd2, dn[2], n.q25);
    n.qx0 = fmaf(w, y.z, n.qx0);
    n.qx1 = fmaf(wd1, y.z, n.qx1);
    n.qx2 = fmaf(wd2, y.z, n.qx2);
    n.qx3 = fmaf(wn0, y.z, n.qx3);
    n.qx4 = fmaf(wn1, y.z, n.qx4);
    n.qx5 = fmaf(wn2, y.z, n.qx5);
}

// Cholesky factorisation + forward / backward substitution of one channel's
// ridge-regularised 6x6 system, in the reference's operation order
// (ops/regression.cu.cc:206-242, 449-467): diagonal pivots
// sqrt(max(1e-5, a_ii - s)), off-diagonals (1/L_jj) * (a_ji - s).
// Lo (nullable) receives the factor, row-major packed lower triangle
// (21 floats per channel), for the backward pass.
//
// FP64 fallback (cond_limit > 0, off by default): when the factor's pivots
// give a condition estimate (max L_ii / min L_ii)^2 above cond_limit, the
// same FP32 normal equations are factored and solved again in double and
// *fallbacks is incremented.  The reference has no such path; with the
// fallback off the result is the reference's.
CD_DEV void solve_fp64(const float (*A)[kP], const float *X, int k, float *beta)
{
    double L[kP][kP];
#pragma unroll
    for (int i = 0; i < kP; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < j; ++q) s = fma(L[i][q], L[j][q], s);
            if (i == j)
                L[i][i] = sqrt(fmax(1e-12, (double)A[i][i] - s));
            else
                L[i][j] = ((double)A[j][i] - s) / L[j][j];
        }
    }
    double Y[kP], bt[kP];
#pragma unroll
    for (int i = 0; i < kP; ++i) {
        double s = X[i];
#pragma unroll
        for (int q = 0; q < i; ++q) s -= L[i][q] * Y[q];
        Y[i] = s / L[i][i];
    }
#pragma unroll
    for (int i = kP - 1; i >= 0; --i) {
        double s = Y[i];
#pragma unroll
        for (int q = i + 1; q < kP; ++q) s -= L[q][i] * bt[q];
        bt[i] = s / L[i][i];
    }
#pragma unroll
    for (int r = 0; r < kP; ++r) beta[r * 3 + k] = (float)bt[r];
}

CD_DEV void solve_channel(const Normal &n, int k, float *beta, float *Lo, float cond_limit = 0.f,
                          unsigned *fallbacks = nullptr)
{
    float A[kP][kP];
    A[0][0] = n.a00; A[0][1] = chan(n.p01, n.q01, k); A[0][2] = chan(n.p02, n.q02, k);
    A[0][3] = n.a03; A[0][4] = n.a04; A[0][5] = n.a05;
    A[1][1] = chan(n.p11, n.q11, k); A[1][2] = chan(n.p12, n.q12, k); A[1][3] = chan(n.p13, n.q13, k);
    A[1][4] = chan(n.p14, n.q14, k); A[1][5] = chan(n.p15, n.q15, k);
    A[2][2] = chan(n.p22, n.q22, k); A[2][3] = chan(n.p23, n.q23, k); A[2][4] = chan(n.p24, n.q24, k);
    A[2][5] = chan(n.p25, n.q25, k);
    A[3][3] = n.a33; A[3][4] = n.a34; A[3][5] = n.a35;
    A[4][4] = n.a44; A[4][5] = n.a45;
    A[5][5] = n.a55;
#pragma unroll
    for (int r = 0; r < kP; ++r) A[r][r] += 1e-3f;
    const float X[kP] = {chan(n.px0, n.qx0, k), chan(n.px1, n.qx1, k), chan(n.px2, n.qx2, k),
                         chan(n.px3, n.qx3, k), chan(n.px4, n.qx4, k), chan(n.px5, n.qx5, k)};
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
    if (Lo) {
#pragma unroll
        for (int i = 0; i < kP; ++i)
#pragma unroll
            for (int j = 0; j <= i; ++j) Lo[21 * k + i * (i + 1) / 2 + j] = L[i][j];
    }
    if (cond_limit > 0.f) {
        float dmin = L[0][0], dmax = L[0][0];
#pragma unroll
        for (int i = 1; i < kP; ++i) {
            dmin = fminf(dmin, L[i][i]);
            dmax = fmaxf(dmax, L[i][i]);
        }
        if (dmax * dmax > cond_limit * (dmin * dmin)) {
            solve_fp64(A, X, k, beta);
            if (fallbacks) atomicAdd(fallbacks, 1u);
            return;
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
// A CTA owns 32 consecutive centres of one centre row; warp 0 solves buffer A
// and warp 1 buffer B, one thread per (centre, buffer), so every centre sums
// its window taps in the reference's order (rows, then columns) with the
// reference's per-tap arithmetic.  The window rows stream through two
// shared-memory row slots (cp.async, double buffered; layout in
// window_rows.cuh): row r + 1 is copied while row r is consumed, and a tap
// is four conflict-free LDS.128.
// ---------------------------------------------------------------------------
constexpr int kCX = kRowCentres;   // centres per CTA
constexpr int kThreads = 64;

// two row slots of 4 float4 groups, then the per-position tables
__host__ __device__ inline size_t regression_smem(int hw, int sp)
{
    const RowGeom g = row_geom(hw, sp);
    return (size_t)2 * 4 * g.npos * sizeof(float4) + (size_t)2 * g.rw * sizeof(int);
}

// exp(x) = 2^(x log2 e) on the ex2.approx.ftz instruction (subnormal results
// flushed to zero).
CD_DEV float exp_ftz(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x * 1.44269504088896341f));
    return y;
}

// Launch bound 7 CTAs per SM: the compiler still fits 128 registers (8 CTAs
// per SM reside) and schedules the one-time solve with fewer spills than
// under a bound of 8 (603 against 613 us per 1920x1080 cross-regression).
__global__ void __launch_bounds__(kThreads, 7) regression_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ vara, const float *__restrict__ varb,
    const float *__restrict__ sda, const float *__restrict__ sdb, float *__restrict__ beta,
    float *__restrict__ chol, float cond_limit, unsigned *__restrict__ fallbacks, int H, int W, int hw, int sp)
{
    extern __shared__ float4 sm4[];
    const RowGeom g = row_geom(hw, sp);
    const int slot = 4 * g.npos;                                   // float4s per slot
    int *pos_gx = reinterpret_cast<int *>(sm4 + 2 * slot);
    int *pos_dst = pos_gx + g.rw;
    const int Ws = W / sp, Hs = H / sp;
    const int b = blockIdx.z;
    const size_t px = (size_t)H * W;
    imga += 3 * px * b;
    imgb += 3 * px * b;
    albedo += 3 * px * b;
    normal += 3 * px * b;
    vara += px * b;
    varb += px * b;
    sda += px * b;
    sdb += px * b;

    const int i0 = blockIdx.x * kCX;
    const int cy = blockIdx.y * sp;
    const int x0 = i0 * sp - hw;
    const int buf = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int R = 2 * hw + 1;

    row_positions(pos_gx, pos_dst, g, x0, W, sp, threadIdx.x, kThreads);
    __syncthreads();

    auto stage = [&](int r, int s) {
        stage_window_row(reinterpret_cast<float *>(sm4 + s * slot), g, pos_gx, pos_dst,
                         clampi(mirror(cy - hw + r, H), 0, H - 1), W, imga, imgb, albedo, normal, vara, varb, sda,
                         sdb, threadIdx.x, kThreads);
    };

    stage(0, 0);
    cp_async_commit();

    // centre values, read directly (clamped for lanes past the last centre)
    const int ci = min(i0 + lane, Ws - 1);
    const size_t c = (size_t)cy * W + (size_t)ci * sp;
    const float3 fc = ld3(buf ? imgb : imga, c);
    const float3 alc = ld3(albedo, c), nrc = ld3(normal, c);
    const float vc = __ldg((buf ? varb : vara) + c), sdc = __ldg((buf ? sdb : sda) + c);
    const float al_c[3] = {alc.x, alc.y, alc.z}, nr_c[3] = {nrc.x, nrc.y, nrc.z};
    // groups read by this buffer: own features + variance, target, albedo, normal
    const int gf = buf ? 1 : 0, gy_ = buf ? 0 : 1;

    Normal nm;
    normal_zero(nm);
    for (int r = 0; r < R; ++r) {
        if (r + 1 < R) {
            stage(r + 1, (r + 1) & 1);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float4 *P = sm4 + (r & 1) * slot;
        const float4 *Gf = P + gf * g.npos, *Gy = P + gy_ * g.npos;
        const float4 *Ga = P + 2 * g.npos, *Gn = P + 3 * g.npos;
        int tm = 0, td = 0;
        for (int t = 0; t < R; ++t) {
            const int o = tm * g.q + td + lane;
            const float4 f4 = Gf[o], y4 = Gy[o], a4 = Ga[o], n4 = Gn[o];
            // own standard deviation: sdA rides in g2.w, sdB in g3.w
            const float sdt = buf ? n4.w : a4.w;
            const float da[3] = {a4.x - al_c[0], a4.y - al_c[1], a4.z - al_c[2]};
            const float dn[3] = {n4.x - nr_c[0], n4.y - nr_c[1], n4.z - nr_c[2]};
            normal_tap(nm, make_float3(f4.x, f4.y, f4.z), fc, make_float3(y4.x, y4.y, y4.z), f4.w, vc, sdt,
                       sdc, da, dn);
            if (++tm == sp) {
                tm = 0;
                ++td;
            }
        }
        __syncthreads();
    }

    if (i0 + lane >= Ws) return;
    const size_t nb_img = (size_t)Hs * Ws;
    const size_t cidx = (size_t)b * nb_img + (size_t)blockIdx.y * Ws + (i0 + lane);
    float *bo = beta + (size_t)buf * gridDim.z * nb_img * kBeta + cidx * kBeta;
    float *lo = chol ? chol + ((size_t)buf * gridDim.z * nb_img + cidx) * 63 : nullptr;
    solve_channel(nm, 0, bo, lo, cond_limit, fallbacks);
    solve_channel(nm, 1, bo, lo, cond_limit, fallbacks);
    solve_channel(nm, 2, bo, lo, cond_limit, fallbacks);
}

// ---------------------------------------------------------------------------
// Block reconstruction (ops/regression.cu.cc:289-365).  A CTA owns 32x4
// output pixels.  The centres their windows reach are staged in shared
// memory as 13 float4 records each.  Each thread sums, over the centres of
// its own window (the reference's clamped iDivUp range, in its order),
// w * (beta_c . delta(p, c)) with delta taken as (p - c).  The quotients use
// a reciprocal and a multiply: unlike the regression's normal equations,
// nothing downstream amplifies their last-bit differences.
//
// Buffers A and B share every centre and pixel pair, so their arithmetic
// runs as packed FP32x2 pairs (low lane A, high lane B; same operation
// order and per-lane rounding as the scalar formulation, ops/regression.cu.cc
// :465-500).  Record of a centre (pairs (A, B) unless noted):
//   0..8   coefficients j = r * 3 + ch, two per record: (A_j, B_j, A_j+1, B_j+1)
//   9      (feature.x, feature.y)      10  (feature.z, variance)
//   11     (sd, albedo.x albedo.y)     12  albedo.z normal.xyz (scalars)
// ---------------------------------------------------------------------------
constexpr int kRX = 32, kRY = 4;
constexpr int kRec = 13;   // float4 per staged centre

__host__ __device__ inline int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

__host__ __device__ inline size_t recon_smem(int hw, int sp, int rs)
{
    const int cxmax = ((kRX - 1) * rs + 2 * hw) / sp + 2;
    const int cymax = ((kRY - 1) * rs + 2 * hw) / sp + 2;
    return (size_t)kRec * cxmax * cymax * sizeof(float4);
}

__global__ void __launch_bounds__(kRX * kRY) recon_kernel(
    const float *__restrict__ imga, const float *__restrict__ imgb,
    const float *__restrict__ albedo, const float *__restrict__ normal,
    const float *__restrict__ vara, const float *__restrict__ varb,
    const float *__restrict__ sda, const float *__restrict__ sdb,
    const float *__restrict__ beta, float *__restrict__ outa, float *__restrict__ outb,
    float *__restrict__ state, int H, int W, int hw, int sp, int rs)
{
    using namespace x2;
    extern __shared__ float4 rec[];
    const int Wr = W / rs, Hr = H / rs;
    const int Ws = W / sp, Hs = H / sp;
    const int b = blockIdx.z;
    const size_t px = (size_t)H * W;
    imga += 3 * px * b;
    imgb += 3 * px * b;
    albedo += 3 * px * b;
    normal += 3 * px * b;
    vara += px * b;
    varb += px * b;
    sda += px * b;
    sdb += px * b;
    const size_t nb_img = (size_t)Hs * Ws;
    const float *betaA = beta + (size_t)b * nb_img * kBeta;
    const float *betaB = beta + (size_t)gridDim.z * nb_img * kBeta + (size_t)b * nb_img * kBeta;

    // centres any pixel of this tile can reach (a superset of every
    // per-pixel range below)
    const int ox0 = blockIdx.x * kRX, oy0 = blockIdx.y * kRY;
    const int ox1 = min(ox0 + kRX - 1, Wr - 1), oy1 = min(oy0 + kRY - 1, Hr - 1);
    const int cx_lo = max(0, floordiv(ox0 * rs - hw, sp));
    const int cx_hi = min(Ws - 1, (ox1 * rs + hw) / sp);
    const int cy_lo = max(0, floordiv(oy0 * rs - hw, sp));
    const int cy_hi = min(Hs - 1, (oy1 * rs + hw) / sp);
    const int ncx = cx_hi - cx_lo + 1, ncy = cy_hi - cy_lo + 1;
    const int nc = ncx * ncy;

    const int tid = threadIdx.y * kRX + threadIdx.x;
    for (int e = tid; e < nc * 9; e += kRX * kRY) {
        const int n = e / 9, f = e - 9 * n;
        const int iy = cy_lo + n / ncx, ix = cx_lo + n % ncx;
        const size_t cb = ((size_t)iy * Ws + ix) * kBeta + 2 * f;
        rec[n * kRec + f] = make_float4(__ldg(betaA + cb), __ldg(betaB + cb), __ldg(betaA + cb + 1), __ldg(betaB + cb + 1));
    }
    for (int n = tid; n < nc; n += kRX * kRY) {
        const int iy = cy_lo + n / ncx, ix = cx_lo + n % ncx;
        const size_t t = (size_t)(iy * sp) * W + ix * sp;
        const float3 fa = ld3(imga, t), fb = ld3(imgb, t), al = ld3(albedo, t), nr = ld3(normal, t);
        rec[n * kRec + 9] = make_float4(fa.x, fb.x, fa.y, fb.y);
        rec[n * kRec + 10] = make_float4(fa.z, fb.z, __ldg(vara + t), __ldg(varb + t));
        rec[n * kRec + 11] = make_float4(__ldg(sda + t), __ldg(sdb + t), al.x, al.y);
        rec[n * kRec + 12] = make_float4(al.z, nr.x, nr.y, nr.z);
    }
    __syncthreads();

    const int cx = ox0 + threadIdx.x, cy = oy0 + threadIdx.y;
    if (cx >= Wr || cy >= Hr) return;
    const int pxo = cx * rs, pyo = cy * rs;
    const size_t p = (size_t)pyo * W + pxo;
    const int sx = max(0, idivup(pxo - hw, sp));
    const int ex = min((W - 1) / sp, (pxo + hw) / sp);
    const int sy = max(0, idivup(pyo - hw, sp));
    const int ey = min((H - 1) / sp, (pyo + hw) / sp);

    const float3 fa = ld3(imga, p), fb = ld3(imgb, p), al = ld3(albedo, p), nr = ld3(normal, p);
    const f2 pf_x = pack(fa.x, fb.x), pf_y = pack(fa.y, fb.y), pf_z = pack(fa.z, fb.z);
    const f2 pvar = pack(__ldg(vara + p), __ldg(varb + p)), psd = pack(__ldg(sda + p), __ldg(sdb + p));
    const f2 k1e2 = pack(1e-2f, 1e-2f), k1e4 = pack(1e-4f, 1e-4f), k1e7 = pack(1e-7f, 1e-7f);
    f2 o0 = 0ull, o1 = 0ull, o2 = 0ull, sw = 0ull;   // +0.0f in both lanes
    for (int iy = sy; iy <= ey; ++iy) {
        const int nrow = (iy - cy_lo) * ncx - cx_lo;
        for (int ix = sx; ix <= ex; ++ix) {
            const float4 *R4 = rec + (nrow + ix) * kRec;
            const ulonglong2 *R = reinterpret_cast<const ulonglong2 *>(R4);
            const ulonglong2 F9 = R[9], F10 = R[10], F11 = R[11];
            const float4 L12 = R4[12];
            const float da0 = al.x - lo(F11.y), da1 = al.y - hi(F11.y), da2 = al.z - L12.x;
            const float dn0 = nr.x - L12.y, dn1 = nr.y - L12.z, dn2 = nr.z - L12.w;
            const f2 d0 = sub2(pf_x, F9.x), d1 = sub2(pf_y, F9.y), d2 = sub2(pf_z, F10.x);
            const f2 den_r = add2(add2(psd, F11.x), k1e2);
            const f2 rden = pack(__fdividef(1.f, lo(den_r)), __fdividef(1.f, hi(den_r)));
            const f2 den_w = add2(add2(pvar, F10.y), k1e4);
            const f2 q = mul2(sqnorm2(d0, d1, d2), pack(__fdividef(1.f, lo(den_w)), __fdividef(1.f, hi(den_w))));
            // exp(-q) + 1e-7 with exp as 2^(-q log2 e) on ex2.approx.ftz: the
            // same weight as __expf wherever exp(-q) is a normal float, and
            // where it is not, both round to 1e-7 after the addition
            const f2 w = add2(pack(exp_ftz(-lo(q)), exp_ftz(-hi(q))), k1e7);
            const ulonglong2 c0 = R[0], c1 = R[1], c2 = R[2], c3 = R[3], c4 = R[4], c5 = R[5], c6 = R[6],
                             c7 = R[7], c8 = R[8];
            // coefficient j = r * 3 + ch sits in record j / 2, half j % 2:
            // r 0: c0.x c0.y c1.x | r 1: c1.y c2.x c2.y | r 2: c3.x c3.y c4.x
            // r 3: c4.y c5.x c5.y | r 4: c6.x c6.y c7.x | r 5: c7.y c8.x c8.y
            f2 p0 = c0.x, p1 = c0.y, p2 = c1.x;
            p0 = fma2(c1.y, mul2(d0, rden), p0);
            p1 = fma2(c2.x, mul2(d1, rden), p1);
            p2 = fma2(c2.y, mul2(d2, rden), p2);
            p0 = fma2(c3.x, pack(da0, da0), p0);
            p1 = fma2(c3.y, pack(da1, da1), p1);
            p2 = fma2(c4.x, pack(da2, da2), p2);
            const f2 n0 = pack(dn0, dn0), n1 = pack(dn1, dn1), n2 = pack(dn2, dn2);
            p0 = fma2(c4.y, n0, p0);
            p1 = fma2(c5.x, n0, p1);
            p2 = fma2(c5.y, n0, p2);
            p0 = fma2(c6.x, n1, p0);
            p1 = fma2(c6.y, n1, p1);
            p2 = fma2(c7.x, n1, p2);
            p0 = fma2(c7.y, n2, p0);
            p1 = fma2(c8.x, n2, p1);
            p2 = fma2(c8.y, n2, p2);
            o0 = fma2(w, p0, o0);
            o1 = fma2(w, p1, o1);
            o2 = fma2(w, p2, o2);
            sw = add2(sw, w);
        }
    }
    const float dA = fmaxf(lo(sw), 1e-7f), dB = fmaxf(hi(sw), 1e-7f);
    const size_t o = (size_t)b * Hr * Wr + (size_t)cy * Wr + cx;
    const float3 qa = make_float3(fmaxf(0.f, lo(o0) / dA), fmaxf(0.f, lo(o1) / dA), fmaxf(0.f, lo(o2) / dA));
    const float3 qb = make_float3(fmaxf(0.f, hi(o0) / dB), fmaxf(0.f, hi(o1) / dB), fmaxf(0.f, hi(o2) / dB));
    if (outa) {
        st3(outa, o, qa);
        st3(outb, o, qb);
    }
    if (state) {   // for the backward: the outputs and the weight sums D, [buffer][pixel]
        float4 *S = reinterpret_cast<float4 *>(state);
        S[o] = make_float4(qa.x, qa.y, qa.z, lo(sw));
        S[(size_t)gridDim.z * Hr * Wr + o] = make_float4(qb.x, qb.y, qb.z, hi(sw));
    }
}

}  // namespace

cudaError_t launch_variance(const float *imga, const float *imgb, float *vara, float *varb, float *sda,
                            float *sdb, int B, int H, int W, cudaStream_t st)
{
    dim3 block(kVX, kVY);
    const bool vec = W % 4 == 0 && ((reinterpret_cast<uintptr_t>(imga) | reinterpret_cast<uintptr_t>(imgb)) & 15) == 0;
    if (vec) {
        dim3 grid((W + kVX - 1) / kVX, (H + kVY - 1) / kVY, B);
        variance_kernel<<<grid, block, 0, st>>>(imga, imgb, vara, varb, sda, sdb, H, W);
    } else {
        dim3 grid((W + kVX - 1) / kVX, (H + kVY - 1) / kVY, 2 * B);
        variance_px_kernel<<<grid, block, 0, st>>>(imga, imgb, vara, varb, sda, sdb, H, W);
    }
    return cudaGetLastError();
}

size_t regression_smem_bytes(int win, int sp) { return regression_smem(win / 2, sp); }
size_t recon_smem_bytes(int win, int sp, int rs) { return recon_smem(win / 2, sp, rs); }

cudaError_t launch_regression(const float *imga, const float *imgb, const float *albedo,
                              const float *normal, const float *vara, const float *varb,
                              const float *sda, const float *sdb, float *beta, int B, int H, int W,
                              int win, int sp, cudaStream_t st, float *chol, float cond_limit,
                              unsigned *fallbacks)
{
    const int hw = win / 2;
    const size_t smem = regression_smem(hw, sp);
    cudaError_t e = cudaFuncSetAttribute(regression_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int Ws = W / sp, Hs = H / sp;
    dim3 grid((Ws + kCX - 1) / kCX, Hs, B);
    regression_kernel<<<grid, kThreads, smem, st>>>(imga, imgb, albedo, normal, vara, varb, sda, sdb, beta,
                                                    chol, cond_limit, fallbacks, H, W, hw, sp);
    return cudaGetLastError();
}

cudaError_t launch_recon(const float *imga, const float *imgb, const float *albedo,
                         const float *normal, const float *vara, const float *varb, const float *sda,
                         const float *sdb, const float *beta, float *outa, float *outb, int B, int H,
                         int W, int win, int sp, int rs, cudaStream_t st, float *state)
{
    const int hw = win / 2;
    const size_t smem = recon_smem(hw, sp, rs);
    cudaError_t e = cudaFuncSetAttribute(recon_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int Wr = W / rs, Hr = H / rs;
    dim3 block(kRX, kRY);
    dim3 grid((Wr + kRX - 1) / kRX, (Hr + kRY - 1) / kRY, B);
    recon_kernel<<<grid, block, smem, st>>>(imga, imgb, albedo, normal, vara, varb, sda, sdb, beta, outa,
                                            outb, state, H, W, hw, sp, rs);
    return cudaGetLastError();
}

}  // namespace cd
