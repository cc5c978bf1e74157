/*
 * cd_oracle.c -- CPU restatement of the reference's per-frame hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA kernels
 * and the timed CPU baseline; no product code path links or calls it.
 *
 * Each function restates, in plain single-precision C, the arithmetic of the
 * reference kernel it cites (file:line inside CGLab-GIST/cross-denoiser).
 * Compiled with -ffp-contract=off so that every float operation rounds
 * exactly where this source says; where the GPU compiler may have fused a
 * multiply into an add the choice is a runtime flag (reproject `mode`), pinned
 * against outputs of the reference kernels themselves (tests/golden).
 *
 * All images are NHWC float32.  Batches are independent; the reference
 * kernels cover batch 0 only (ops/regression.cc:190, temporal.cu.cc:76), so
 * parity against it is taken per batch slice.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>

#define ORC_API __attribute__((visibility("default")))

static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }

/* Integer ceil-division with C's truncating '/' and '%', as iDivUp in
   ops/cuda_utils.cuh:275-278 (for negative a it rounds towards +1, e.g.
   iDivUp(-3, 4) == 1). */
static inline int idivup(int a, int b) { return (a % b != 0) ? (a / b + 1) : (a / b); }

/* Reflect-101 index used by the regression and spatial-filter windows
   (ops/regression.cu.cc:128-129, 413-414). */
static inline int mirror(int i, int n) { return (i >= n) ? 2 * n - 2 - i : abs(i); }

/* float -> int truncation as the GPU's cvt.rzi.s32.f32 does it (saturating,
   NaN -> 0); identical to a C cast for in-range values. */
static inline int f2i_trunc(float v)
{
    if (v != v) return 0;
    if (v >= 2147483648.0f) return INT_MAX;
    if (v <= -2147483904.0f) return INT_MIN;
    return (int)v;
}

static inline float norm2_3(float x, float y, float z)
{
    /* x*x + y*y + z*z evaluated left to right (ops/cuda_utils.cuh:171-174) */
    return (x * x + y * y) + z * z;
}

/* ========================================================================= */
/* Variance estimate: EstInputVarianceKernel, ops/regression.cu.cc:244-276    */
/* (winSize fixed to 3 by CrossRegressionFunc, :490-491).                     */
/* ========================================================================= */
static void variance_plane(const float *img, float *var, int H, int W)
{
#pragma omp parallel for schedule(static)
    for (int cy = 0; cy < H; ++cy) {
        for (int cx = 0; cx < W; ++cx) {
            const int sx = imax(0, cx - 1), ex = imin(W - 1, cx + 1);
            const int sy = imax(0, cy - 1), ey = imin(H - 1, cy + 1);
            const int c = cy * W + cx;
            float ax = 0.f, ay = 0.f, az = 0.f;
            int n = 0;
            for (int iy = sy; iy <= ey; ++iy)
                for (int ix = sx; ix <= ex; ++ix) {
                    const int i = iy * W + ix;
                    if (i != c) {
                        ax += img[3 * i + 0];
                        ay += img[3 * i + 1];
                        az += img[3 * i + 2];
                        ++n;
                    }
                }
            const float fn = (float)n;
            const float dx = ax / fn - img[3 * c + 0];
            const float dy = ay / fn - img[3 * c + 1];
            const float dz = az / fn - img[3 * c + 2];
            var[c] = norm2_3(dx, dy, dz);
        }
    }
}

ORC_API void orc_variance(const float *img, float *var, int B, int H, int W)
{
    for (int b = 0; b < B; ++b)
        variance_plane(img + (size_t)b * H * W * 3, var + (size_t)b * H * W, H, W);
}

/* ========================================================================= */
/* Per-centre weighted least squares: RegressionKernel, cholesky_color and    */
/* forward_backward_solver, ops/regression.cu.cc:206-242, 278-287, 367-475.   */
/* ========================================================================= */
#define P 6

static void cholesky_solve_channel(float A[P][P], const float XtB[P], float beta[P])
{
    float L[P][P];
    memset(L, 0, sizeof(L));
    for (int i = 0; i < P; ++i) {
        for (int j = 0; j < i + 1; ++j) {
            float s = 0.f;
            for (int k = 0; k < j; ++k) s = fmaf(L[i][k], L[j][k], s);
            if (i == j)
                L[i][j] = sqrtf(fmaxf(1e-5f, A[i][i] - s));
            else
                L[i][j] = (1.f / L[j][j]) * (A[j][i] - s);
        }
    }
    float Wv[P];
    Wv[0] = XtB[0] / L[0][0];
    for (int i = 1; i < P; ++i) {
        float s = 0.f;
        for (int k = 0; k < i; ++k) s = fmaf(L[i][k], Wv[k], s);
        Wv[i] = (XtB[i] - s) / L[i][i];
    }
    beta[P - 1] = Wv[P - 1] / L[P - 1][P - 1];
    for (int i = P - 2; i >= 0; --i) {
        float s = 0.f;
        for (int k = P - 1; k > i; --k) s = fmaf(L[k][i], beta[k], s);
        beta[i] = (Wv[i] - s) / L[i][i];
    }
}

/* beta layout: [centre][6][3] (coefficient-major, channel-minor). */
static void regress_plane(const float *y_img, const float *f_img, const float *var,
                          const float *alb, const float *nrm, float *beta,
                          int H, int W, int win, int sp)
{
    const int hw = win / 2;
    const int Hs = H / sp, Ws = W / sp;
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = 0; j < Hs; ++j) {
        for (int i = 0; i < Ws; ++i) {
            const int cx = i * sp, cy = j * sp;
            const int c = cy * W + cx;
            const float cf[3] = {f_img[3 * c], f_img[3 * c + 1], f_img[3 * c + 2]};
            const float ca[3] = {alb[3 * c], alb[3 * c + 1], alb[3 * c + 2]};
            const float cn[3] = {nrm[3 * c], nrm[3 * c + 1], nrm[3 * c + 2]};
            const float cVar = var[c];
            const float cStd = sqrtf(cVar);
            float A[3][P][P];
            float X[3][P];
            memset(A, 0, sizeof(A));
            memset(X, 0, sizeof(X));
            for (int iy = cy - hw; iy <= cy + hw; ++iy) {
                for (int ix = cx - hw; ix <= cx + hw; ++ix) {
                    const int t = mirror(iy, H) * W + mirror(ix, W);
                    const float iVar = var[t];
                    const float iStd = sqrtf(iVar);
                    const float den = (cStd + iStd) + 1e-2f;
                    const float df[3] = {f_img[3 * t] - cf[0], f_img[3 * t + 1] - cf[1], f_img[3 * t + 2] - cf[2]};
                    const float dist = norm2_3(df[0], df[1], df[2]) / ((cVar + iVar) + 1e-4f);
                    const float w = expf(-dist) + 1e-7f;
                    for (int ch = 0; ch < 3; ++ch) {
                        float d[P];
                        d[0] = 1.f;
                        d[1] = df[ch] / den;
                        d[2] = alb[3 * t + ch] - ca[ch];
                        d[3] = nrm[3 * t + 0] - cn[0];
                        d[4] = nrm[3 * t + 1] - cn[1];
                        d[5] = nrm[3 * t + 2] - cn[2];
                        const float yv = y_img[3 * t + ch];
                        for (int r = 0; r < P; ++r) {
                            const float wr = w * d[r];
                            for (int q = r; q < P; ++q) A[ch][r][q] = fmaf(wr, d[q], A[ch][r][q]);
                            X[ch][r] = fmaf(wr, yv, X[ch][r]);
                        }
                    }
                }
            }
            float *bout = beta + (size_t)(j * Ws + i) * P * 3;
            for (int ch = 0; ch < 3; ++ch) {
                for (int r = 0; r < P; ++r)
                    for (int q = 0; q < r; ++q) A[ch][r][q] = A[ch][q][r];
                for (int r = 0; r < P; ++r) A[ch][r][r] += 1e-3f;
                float bc[P];
                cholesky_solve_channel(A[ch], X[ch], bc);
                for (int r = 0; r < P; ++r) bout[r * 3 + ch] = bc[r];
            }
        }
    }
}

/* BlockRecon, ops/regression.cu.cc:289-365. */
static void recon_plane(const float *f_img, const float *var, const float *alb,
                        const float *nrm, const float *beta, float *out,
                        int H, int W, int win, int sp, int rs)
{
    const int hw = win / 2;
    const int Wr = W / rs, Hr = H / rs;
    const int Wb = W / sp;
#pragma omp parallel for schedule(static)
    for (int cy = 0; cy < Hr; ++cy) {
        for (int cx = 0; cx < Wr; ++cx) {
            const int px = cx * rs, py = cy * rs;
            const int p = py * W + px;
            const int sx = imax(0, idivup(px - hw, sp));
            const int ex = imin((W - 1) / sp, (px + hw) / sp);
            const int sy = imax(0, idivup(py - hw, sp));
            const int ey = imin((H - 1) / sp, (py + hw) / sp);
            const float pf[3] = {f_img[3 * p], f_img[3 * p + 1], f_img[3 * p + 2]};
            const float pa[3] = {alb[3 * p], alb[3 * p + 1], alb[3 * p + 2]};
            const float pn[3] = {nrm[3 * p], nrm[3 * p + 1], nrm[3 * p + 2]};
            const float pVar = var[p];
            const float pStd = sqrtf(pVar);
            float o[3] = {0.f, 0.f, 0.f};
            float sumW = 0.f;
            for (int iy = sy; iy <= ey; ++iy) {
                for (int ix = sx; ix <= ex; ++ix) {
                    const float *bc = beta + (size_t)(iy * Wb + ix) * P * 3;
                    const int t = (iy * sp) * W + ix * sp;
                    const float iVar = var[t];
                    const float iStd = sqrtf(iVar);
                    const float den = (pStd + iStd) + 1e-2f;
                    const float df[3] = {pf[0] - f_img[3 * t], pf[1] - f_img[3 * t + 1], pf[2] - f_img[3 * t + 2]};
                    const float dn[3] = {pn[0] - nrm[3 * t], pn[1] - nrm[3 * t + 1], pn[2] - nrm[3 * t + 2]};
                    float pred[3];
                    for (int ch = 0; ch < 3; ++ch) {
                        const float d[P] = {1.f, df[ch] / den, pa[ch] - alb[3 * t + ch], dn[0], dn[1], dn[2]};
                        float s = 0.f;
                        for (int r = 0; r < P; ++r) s = fmaf(bc[r * 3 + ch], d[r], s);
                        pred[ch] = s;
                    }
                    /* regressionWgt(cColWgt=f(p), iColWgt=f(c), ...): norm2(f(c) - f(p)) */
                    const float dist = norm2_3(-df[0], -df[1], -df[2]) / ((pVar + iVar) + 1e-4f);
                    const float w = expf(-dist) + 1e-7f;
                    for (int ch = 0; ch < 3; ++ch) o[ch] = fmaf(w, pred[ch], o[ch]);
                    sumW += w;
                }
            }
            const float den = fmaxf(sumW, 1e-7f);
            float *op = out + (size_t)(cy * Wr + cx) * 3;
            for (int ch = 0; ch < 3; ++ch) op[ch] = fmaxf(0.f, o[ch] / den);
        }
    }
}

/* CrossRegressionFunc, ops/regression.cu.cc:477-500: var(A), var(B),
   beta_A = regress(y=imgb | features imga), beta_B = regress(y=imga | imgb),
   outa = recon(beta_A, imga), outb = recon(beta_B, imgb).
   betaA/betaB may be NULL (scratch is then allocated here). */
ORC_API void orc_cross_regression(const float *imga, const float *imgb,
                                  const float *albedo, const float *normal,
                                  float *outa, float *outb, float *vara, float *varb,
                                  float *betaA, float *betaB,
                                  int B, int H, int W, int win, int sp, int rs)
{
    const size_t px = (size_t)H * W;
    const size_t nbeta = (size_t)(H / sp) * (W / sp) * P * 3;
    float *ba = betaA ? NULL : (float *)malloc(nbeta * sizeof(float));
    float *bb = betaB ? NULL : (float *)malloc(nbeta * sizeof(float));
    for (int b = 0; b < B; ++b) {
        const float *ia = imga + b * px * 3, *ib = imgb + b * px * 3;
        const float *al = albedo + b * px * 3, *nr = normal + b * px * 3;
        float *va = vara + b * px, *vb = varb + b * px;
        float *bA = betaA ? betaA + b * nbeta : ba;
        float *bB = betaB ? betaB + b * nbeta : bb;
        const size_t opx = (size_t)(H / rs) * (W / rs) * 3;
        variance_plane(ia, va, H, W);
        variance_plane(ib, vb, H, W);
        regress_plane(ib, ia, va, al, nr, bA, H, W, win, sp);
        regress_plane(ia, ib, vb, al, nr, bB, H, W, win, sp);
        recon_plane(ia, va, al, nr, bA, outa + b * opx, H, W, win, sp, rs);
        recon_plane(ib, vb, al, nr, bB, outb + b * opx, H, W, win, sp, rs);
    }
    free(ba);
    free(bb);
}

/* ========================================================================= */
/* Spatial filter forward, SpatialFilterKernel ops/regression.cu.cc:84-195.   */
/* partA/partB (nullable) receive the reference's per-pixel band partials,    */
/* 4 x (x,y,z,w) per pixel = 16 floats (the gradBandA/B scratch).             */
/* ========================================================================= */
ORC_API void orc_spatial_filter(const float *imga, const float *imgb, const float *albedo,
                                const float *normal, const float *band,
                                float *acca, float *accb, float *wsa, float *wsb,
                                float *partA, float *partB,
                                int B, int H, int W, int win)
{
    const int hw = win / 2;
    const size_t px = (size_t)H * W;
    for (int b = 0; b < B; ++b) {
        const float *ia = imga + b * px * 3, *ib = imgb + b * px * 3;
        const float *al = albedo + b * px * 3, *nr = normal + b * px * 3;
        const float *bd = band + b * px * 5;
#pragma omp parallel for schedule(static)
        for (int cy = 0; cy < H; ++cy) {
            for (int cx = 0; cx < W; ++cx) {
                const int c = cy * W + cx;
                const float *cb = bd + 5 * c;
                float aA[3] = {0, 0, 0}, aB[3] = {0, 0, 0}, sA = 0.f, sB = 0.f;
                float gA[4][4], gB[4][4];
                memset(gA, 0, sizeof(gA));
                memset(gB, 0, sizeof(gB));
                for (int iy = cy - hw; iy <= cy + hw; ++iy) {
                    for (int ix = cx - hw; ix <= cx + hw; ++ix) {
                        const int t = mirror(iy, H) * W + mirror(ix, W);
                        const float dy = (float)(cy - iy) / (float)hw;
                        const float dx = (float)(cx - ix) / (float)hw;
                        const float pd = dx * dx + dy * dy;
                        const float dA = norm2_3(ia[3 * c] - ia[3 * t], ia[3 * c + 1] - ia[3 * t + 1], ia[3 * c + 2] - ia[3 * t + 2]);
                        const float dB = norm2_3(ib[3 * c] - ib[3 * t], ib[3 * c + 1] - ib[3 * t + 1], ib[3 * c + 2] - ib[3 * t + 2]);
                        const float dAl = norm2_3(al[3 * c] - al[3 * t], al[3 * c + 1] - al[3 * t + 1], al[3 * c + 2] - al[3 * t + 2]);
                        const float dN = norm2_3(nr[3 * c] - nr[3 * t], nr[3 * c + 1] - nr[3 * t + 1], nr[3 * c + 2] - nr[3 * t + 2]);
                        const float eA = ((-cb[0] * dA - cb[2] * dAl) - cb[3] * dN) - cb[4] * pd;
                        const float eB = ((-cb[1] * dB - cb[2] * dAl) - cb[3] * dN) - cb[4] * pd;
                        const float wA = expf(eA), wB = expf(eB);
                        for (int k = 0; k < 3; ++k) {
                            aA[k] = fmaf(wA, ia[3 * t + k], aA[k]);
                            aB[k] = fmaf(wB, ib[3 * t + k], aB[k]);
                        }
                        sA += wA;
                        sB += wB;
                        if (partA) {
                            const float dk[4] = {dA, dAl, dN, pd};
                            const float dkB[4] = {dB, dAl, dN, pd};
                            for (int k = 0; k < 4; ++k) {
                                const float da = wA * (-dk[k]);
                                const float db = wB * (-dkB[k]);
                                for (int q = 0; q < 3; ++q) {
                                    gA[k][q] = fmaf(da, ia[3 * t + q], gA[k][q]);
                                    gB[k][q] = fmaf(db, ib[3 * t + q], gB[k][q]);
                                }
                                gA[k][3] += da;
                                gB[k][3] += db;
                            }
                        }
                    }
                }
                const size_t o = b * px + c;
                for (int k = 0; k < 3; ++k) {
                    acca[o * 3 + k] = aA[k];
                    accb[o * 3 + k] = aB[k];
                }
                wsa[o] = sA;
                wsb[o] = sB;
                if (partA) {
                    for (int k = 0; k < 4; ++k)
                        for (int q = 0; q < 4; ++q) {
                            partA[o * 16 + k * 4 + q] = gA[k][q];
                            partB[o * 16 + k * 4 + q] = gB[k][q];
                        }
                }
            }
        }
    }
}

/* Spatial filter gradient from stored partials, SpatialFilterGradKernel
   ops/regression.cu.cc:33-81.  gband[0] from A only, [1] from B only,
   [2..4] = A + B. */
ORC_API void orc_spatial_filter_grad(const float *g_acca, const float *g_accb,
                                     const float *g_wsa, const float *g_wsb,
                                     const float *partA, const float *partB,
                                     float *gband, int B, int H, int W)
{
    const size_t n = (size_t)B * H * W;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) {
        float oa[4], ob[4];
        for (int k = 0; k < 4; ++k) {
            const float *pa = partA + i * 16 + k * 4, *pb = partB + i * 16 + k * 4;
            oa[k] = ((g_acca[3 * i] * pa[0] + g_acca[3 * i + 1] * pa[1]) + g_acca[3 * i + 2] * pa[2]) + g_wsa[i] * pa[3];
            ob[k] = ((g_accb[3 * i] * pb[0] + g_accb[3 * i + 1] * pb[1]) + g_accb[3 * i + 2] * pb[2]) + g_wsb[i] * pb[3];
        }
        gband[5 * i + 0] = oa[0];
        gband[5 * i + 1] = ob[0];
        gband[5 * i + 2] = oa[1] + ob[1];
        gband[5 * i + 3] = oa[2] + ob[2];
        gband[5 * i + 4] = oa[3] + ob[3];
    }
}

/* ========================================================================= */
/* Reprojection: isReprojValid + Reproject, ops/reproject.cu.cc:32-238.       */
/*                                                                            */
/* `mode` selects how the float expressions that a GPU compiler may contract  */
/* are rounded (all other operations round exactly as written):               */
/*   bit 0  iposPrev = fma(mvec, dim, pos) + 0.5     (else pos + mvec*dim)    */
/*   bit 1  posPrev  = fma(mvec, dim, floor(pos))    (else floor(pos)+mvec*dim)*/
/*   bits 2-3  |n - n'|^2: 0 = ((xx+yy)+zz), 1 = fma(z,z,fma(x,x,yy)),        */
/*             2 = fma(z,z,fma(y,y,xx)), 3 = fma(z,z,xx+yy)                   */
/*   bit 4  bilinear weight sum accumulated with fma                          */
/* ========================================================================= */
#define ORC_RP_FMA_IPOS 1
#define ORC_RP_FMA_POSPREV 2
#define ORC_RP_DOT_SHIFT 2
#define ORC_RP_FMA_SUMW 16

static inline float dot_mode(float x, float y, float z, int m)
{
    switch (m) {
    case 1: return fmaf(z, z, fmaf(x, x, y * y));
    case 2: return fmaf(z, z, fmaf(y, y, x * x));
    case 3: return fmaf(z, z, x * x + y * y);
    default: return (x * x + y * y) + z * z;
    }
}

static inline int reproj_valid(int W, int H, int ipx, int ipy, float Z, float Zp, float fwZ,
                               const float *n, const float *np, float fwN, int mode)
{
    if (ipx < 1 || ipy < 1 || ipx > W - 1 || ipy > H - 1) return 0;
    if (fabsf(Zp - Z) / (fwZ + 1e-2f) > 10.f) return 0;
    const float dist = sqrtf(dot_mode(n[0] - np[0], n[1] - np[1], n[2] - np[2],
                                      (mode >> ORC_RP_DOT_SHIFT) & 3));
    if ((double)dist / ((double)fwN + 1e-2) > 4.0) return 0;
    return 1;
}

ORC_API void orc_reproject(const float *mvec, int n_list, const float *const *inputs,
                           const int *channels, float *const *outputs,
                           const float *linz, const float *plinz, const float *nrm,
                           const float *pnrm, const float *pnfw, const float *opac,
                           const float *popac, uint8_t *success,
                           int B, int H, int W, int mode)
{
    static const int ox[4] = {0, 1, 0, 1}, oy[4] = {0, 0, 1, 1};
    const size_t px = (size_t)H * W;
    for (int b = 0; b < B; ++b) {
        const size_t base = b * px;
#pragma omp parallel for schedule(static)
        for (int cy = 0; cy < H; ++cy) {
            for (int cx = 0; cx < W; ++cx) {
                const size_t c = base + (size_t)cy * W + cx;
                for (int d = 0; d < n_list; ++d)
                    for (int k = 0; k < channels[d]; ++k) outputs[d][c * channels[d] + k] = 0.f;
                if (opac[c] == 0.f) {
                    success[c] = 0;
                    continue;
                }
                const float mx = mvec[3 * c], my = mvec[3 * c + 1];
                const float fwN = pnfw[3 * c + 1];
                const float fx = (float)cx, fy = (float)cy, fW = (float)W, fH = (float)H;
                float ux, uy;
                if (mode & ORC_RP_FMA_IPOS) {
                    ux = fmaf(mx, fW, fx);
                    uy = fmaf(my, fH, fy);
                } else {
                    ux = fx + mx * fW;
                    uy = fy + my * fH;
                }
                const int ipx = f2i_trunc(ux + 0.5f), ipy = f2i_trunc(uy + 0.5f);
                const float Z = linz[3 * c], fwZ = linz[3 * c + 1];
                const float n[3] = {nrm[3 * c], nrm[3 * c + 1], nrm[3 * c + 2]};
                float ppx, ppy;
                if (mode & ORC_RP_FMA_POSPREV) {
                    ppx = fmaf(mx, fW, floorf(fx));
                    ppy = fmaf(my, fH, floorf(fy));
                } else {
                    ppx = floorf(fx) + mx * fW;
                    ppy = floorf(fy) + my * fH;
                }
                const int lx = f2i_trunc(ppx), ly = f2i_trunc(ppy);
                int v[4];
                int valid = 0;
                for (int s = 0; s < 4; ++s) {
                    const int qx = lx + ox[s], qy = ly + oy[s];
                    if (qx >= W || qx < 0 || qy >= H || qy < 0 || popac[base + (size_t)qy * W + qx] == 0.f) {
                        v[s] = 0;
                    } else {
                        const size_t q = base + (size_t)qy * W + qx;
                        v[s] = reproj_valid(W, H, ipx, ipy, Z, plinz[3 * q], fwZ, n, pnrm + 3 * q, fwN, mode);
                        valid = valid || v[s];
                    }
                }
                if (valid) {
                    const float x = ppx - floorf(ppx), y = ppy - floorf(ppy);
                    const float a0 = 1.f - x, a1 = x, b0 = 1.f - y, b1 = y;
                    const float fa[4] = {a0, a1, a0, a1}, fb[4] = {b0, b0, b1, b1};
                    float wgt[4];
                    for (int s = 0; s < 4; ++s) wgt[s] = fa[s] * fb[s];
                    float sumw = 0.f;
                    for (int s = 0; s < 4; ++s) {
                        if (!v[s]) continue;
                        const size_t q = base + (size_t)(ly + oy[s]) * W + (lx + ox[s]);
                        for (int d = 0; d < n_list; ++d)
                            for (int k = 0; k < channels[d]; ++k) {
                                float *o = &outputs[d][c * channels[d] + k];
                                *o = fmaf(wgt[s], inputs[d][q * channels[d] + k], *o);
                            }
                        sumw = (mode & ORC_RP_FMA_SUMW) ? fmaf(fa[s], fb[s], sumw) : sumw + wgt[s];
                    }
                    valid = (sumw >= 0.01f);
                    for (int d = 0; d < n_list; ++d)
                        for (int k = 0; k < channels[d]; ++k) {
                            float *o = &outputs[d][c * channels[d] + k];
                            *o = valid ? *o / sumw : 0.f;
                        }
                }
                if (!valid) {
                    float nValid = 0.f;
                    for (int yy = -1; yy <= 1; ++yy) {
                        for (int xx = -1; xx <= 1; ++xx) {
                            const int qx = ipx + xx, qy = ipy + yy;
                            /* the reference reads prev_opacity here without the
                               batch offset (ops/reproject.cu.cc:191) */
                            if (qx >= W || qx < 0 || qy >= H || qy < 0 || popac[(size_t)qy * W + qx] == 0.f)
                                continue;
                            const size_t q = base + (size_t)qy * W + qx;
                            if (reproj_valid(W, H, ipx, ipy, Z, plinz[3 * q], fwZ, n, pnrm + 3 * q, fwN, mode)) {
                                for (int d = 0; d < n_list; ++d)
                                    for (int k = 0; k < channels[d]; ++k)
                                        outputs[d][c * channels[d] + k] += inputs[d][q * channels[d] + k];
                                nValid += 1.f;
                            }
                        }
                    }
                    if (nValid > 0.f) {
                        valid = 1;
                        for (int d = 0; d < n_list; ++d)
                            for (int k = 0; k < channels[d]; ++k) outputs[d][c * channels[d] + k] /= nValid;
                    }
                }
                if (!valid)
                    for (int d = 0; d < n_list; ++d)
                        for (int k = 0; k < channels[d]; ++k) outputs[d][c * channels[d] + k] = 0.f;
                success[c] = (uint8_t)valid;
            }
        }
    }
}

/* ========================================================================= */
/* 3x3 erosion with SAME padding (scripts/main.py:270-276).                   */
/* ========================================================================= */
ORC_API void orc_erode3x3(const uint8_t *success, float *out, int B, int H, int W)
{
    const size_t px = (size_t)H * W;
    for (int b = 0; b < B; ++b) {
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                float m = 1.f;
                for (int yy = imax(0, y - 1); yy <= imin(H - 1, y + 1); ++yy)
                    for (int xx = imax(0, x - 1); xx <= imin(W - 1, x + 1); ++xx)
                        m = fminf(m, success[b * px + (size_t)yy * W + xx] ? 1.f : 0.f);
                out[b * px + (size_t)y * W + x] = m;
            }
    }
}

/* ========================================================================= */
/* Temporal screening: fo2 + TemporalScreening, ops/temporal.cu.cc:28-198.   */
/* ========================================================================= */
#define ORC_TS_BIG 10000000.f

ORC_API void orc_temporal_screening(const float *cur1, const float *cur2, const float *prev,
                                    const float *prev1, const float *prev2, const float *rs,
                                    float *out, float *out1, float *out2, float *succ,
                                    int B, int H, int W, int win_curr, int win_prev)
{
    const size_t px = (size_t)H * W;
    const int hc = win_curr / 2, hp = win_prev / 2;
    for (int b = 0; b < B; ++b) {
        const float *c1 = cur1 + b * px * 3, *c2 = cur2 + b * px * 3;
        const float *pv = prev + b * px * 3, *p1 = prev1 + b * px * 3, *p2 = prev2 + b * px * 3;
        const float *r = rs + b * px;
        float *o = out + b * px * 3, *o1 = out1 + b * px * 3, *o2 = out2 + b * px * 3;
        float *sc = succ + b * px;
#pragma omp parallel for schedule(static)
        for (int cy = 0; cy < H; ++cy) {
            for (int cx = 0; cx < W; ++cx) {
                const int c = cy * W + cx;
                float cu[3], a1[3], a2[3];
                for (int k = 0; k < 3; ++k) {
                    a1[k] = c1[3 * c + k];
                    a2[k] = c2[3 * c + k];
                    cu[k] = (a1[k] + a2[k]) * 0.5f;
                }
                if (r[c] + 1e-4f < 1.f) {
                    for (int k = 0; k < 3; ++k) {
                        o[3 * c + k] = cu[k];
                        o1[3 * c + k] = a1[k];
                        o2[3 * c + k] = a2[k];
                    }
                    sc[c] = 0.f;
                    continue;
                }
                float mnC[3], mxC[3], mnC1[3], mxC1[3], mnC2[3], mxC2[3];
                float mnP[3], mxP[3], mnP1[3], mxP1[3], mnP2[3], mxP2[3];
                for (int k = 0; k < 3; ++k) {
                    mnC[k] = mnC1[k] = mnC2[k] = mnP[k] = mnP1[k] = mnP2[k] = ORC_TS_BIG;
                    mxC[k] = mxC1[k] = mxC2[k] = mxP[k] = mxP1[k] = mxP2[k] = -ORC_TS_BIG;
                }
                for (int iy = cy - hc; iy <= cy + hc; ++iy)
                    for (int ix = cx - hc; ix <= cx + hc; ++ix) {
                        if (ix < 0 || ix >= W || iy < 0 || iy >= H) continue;
                        const int i = iy * W + ix;
                        for (int k = 0; k < 3; ++k) {
                            const float v1 = c1[3 * i + k], v2 = c2[3 * i + k];
                            const float v = (v1 + v2) * 0.5f;
                            mnC1[k] = fminf(mnC1[k], v1);
                            mxC1[k] = fmaxf(mxC1[k], v1);
                            mnC2[k] = fminf(mnC2[k], v2);
                            mxC2[k] = fmaxf(mxC2[k], v2);
                            mnC[k] = fminf(mnC[k], v);
                            mxC[k] = fmaxf(mxC[k], v);
                        }
                    }
                for (int iy = cy - hp; iy <= cy + hp; ++iy)
                    for (int ix = cx - hp; ix <= cx + hp; ++ix) {
                        if (ix < 0 || ix >= W || iy < 0 || iy >= H) continue;
                        const int i = iy * W + ix;
                        if (r[i] < 1.f) continue;
                        for (int k = 0; k < 3; ++k) {
                            mnP[k] = fminf(mnP[k], pv[3 * i + k]);
                            mxP[k] = fmaxf(mxP[k], pv[3 * i + k]);
                            mnP1[k] = fminf(mnP1[k], p1[3 * i + k]);
                            mxP1[k] = fmaxf(mxP1[k], p1[3 * i + k]);
                            mnP2[k] = fminf(mnP2[k], p2[3 * i + k]);
                            mxP2[k] = fmaxf(mxP2[k], p2[3 * i + k]);
                        }
                    }
#define ALL_LESS(a, b) ((a)[0] < (b)[0] && (a)[1] < (b)[1] && (a)[2] < (b)[2])
                const int s0 = ALL_LESS(mnP, mxC) && ALL_LESS(mnC, mxP);
                const int s1 = ALL_LESS(mnP1, mxC1) && ALL_LESS(mnC1, mxP1);
                const int s2 = ALL_LESS(mnP2, mxC2) && ALL_LESS(mnC2, mxP2);
#undef ALL_LESS
                for (int k = 0; k < 3; ++k) {
                    o[3 * c + k] = s0 ? pv[3 * c + k] : cu[k];
                    o1[3 * c + k] = s1 ? p1[3 * c + k] : a1[k];
                    o2[3 * c + k] = s2 ? p2[3 * c + k] : a2[k];
                }
                sc[c] = s0 ? 1.f : 0.f;
            }
        }
    }
}
