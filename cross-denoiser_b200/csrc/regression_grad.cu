// Gradient of CrossRegression with respect to its four images.
//
// The reference registers no gradient for this op (scripts/ops.py:23-32);
// this is the analytic derivative of the forward of regression.cu
// (ops/regression.cu.cc:244-500 semantics), for dL/d(outa, outb, vara, varb)
// given.  Per buffer (A: features f = imga, target y = imgb; B: f = imgb,
// y = imga), with s = sqrt(v):
//
//   regression   delta_t = [1, (f_t-f_c)/(s_c+s_t+0.01), alb_t-alb_c, n_t-n_c]
//                w_t = exp(-|f_t-f_c|^2/(v_c+v_t+1e-4)) + 1e-7
//                A = sum_t w delta delta^T + 1e-3 I,  b = sum_t w delta y_t,  beta = A^-1 b
//   recon        out_p = max(0, N_p / max(D_p, 1e-7)),  N_p = sum_c w'_pc beta_c . delta'_pc,
//                D_p = sum_c w'_pc  (delta', w' as above with (p - c) ordering)
//
// Backward of beta = A^-1 b, with u = A^-1 dL/dbeta, a = u . delta,
// r = y_t - beta . delta (the residual at the tap):
//   dL/dw_t = a r,   dL/ddelta_t = w (u r - a beta),   dL/dy_t = w a.
// The Cholesky pivot clamp max(1e-5, .) of the reference never binds for
// the ridge-regularised systems and is treated as the identity; s = 0
// (v = 0) contributes no gradient through sqrt.
//
// Passes (each pixel or centre is written by exactly one thread per pass;
// passes are stream ordered, so no atomics):
//   1. variance + std, forward regression keeping each centre's Cholesky factor
//   2. recon backward, pixel side (dL/dN, dL/dD stored per output pixel)
//   3. recon backward, centre side (dL/dbeta)
//   4. solve backward (u) and the regression's centre-side terms
//   5. the regression's tap-side terms, gathered per pixel over every
//      (centre, window position) whose reflect-101 image is that pixel
//   6. sqrt / variance chain and assembly of dL/dimga, dL/dimgb, dL/dalbedo,
//      dL/dnormal.
#include <cuda_runtime.h>
#include "cd_common.cuh"

namespace cd {
namespace {

constexpr int kP = 6, kBeta = 18, kL = 63;

struct GBuf {
    const float *f, *y, *v, *s, *beta, *L;
    float *u, *gbeta, *gN, *gD, *gf, *gy, *gs, *gv, *hn;
    const float *gout, *gvar;   // upstream dL/dout [R,3], dL/dvar [P] (nullable)
};

struct GArgs {
    GBuf bf[2];
    const float *alb, *nrm;
    float *galb, *gn;
    float *out_a, *out_b, *out_alb, *out_n;   // final gradients
    int H, W, hw, sp, rs, Hs, Ws, Hr, Wr;
};

CD_DEV float3 f3(const float *p, size_t i) { return ld3(p, i); }
CD_DEV void add3(float *p, size_t i, float3 v)
{
    p[3 * i] += v.x;
    p[3 * i + 1] += v.y;
    p[3 * i + 2] += v.z;
}

// Pixel-centre pair of the reconstruction (p - c ordering) and its
// derivatives with respect to the pair's inputs, given dL/dN (gN) and dL/dD.
struct PairGrad {
    float pred[3], w;
    float3 gdf;        // dL/d(f_p - f_c)
    float gden, gV;    // dL/d(s_p + s_c + 0.01), dL/d(v_p + v_c + 1e-4)
    float3 gda, gdn;   // dL/d(alb_p - alb_c), dL/d(n_p - n_c)
    float gbeta[kBeta];
};

template <bool kNeedBeta>
CD_DEV void recon_pair(float3 fp, float3 fc, float sp_, float sc, float vp, float vc, float3 da, float3 dn,
                       const float *beta, const float gN[3], float gD, PairGrad &g)
{
    const float df[3] = {fp.x - fc.x, fp.y - fc.y, fp.z - fc.z};
    const float dav[3] = {da.x, da.y, da.z}, dnv[3] = {dn.x, dn.y, dn.z};
    const float den = (sp_ + sc) + 1e-2f;
    const float V = (vp + vc) + 1e-4f;
    // the pair's quotients share two denominators (den >= 1e-2, V >= 1e-4):
    // one reciprocal each (about 2 ulp) instead of a division per quotient
    const float rden = __fdividef(1.f, den), rV = __fdividef(1.f, V);
    const float dist = (df[0] * df[0] + df[1] * df[1] + df[2] * df[2]) * rV;
    const float e = __expf(-dist);
    g.w = e + 1e-7f;
    float gw = gD, gd1[3], gdn[3] = {0.f, 0.f, 0.f}, d1[3];
    float gda_[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        d1[k] = df[k] * rden;
        const float *bk = beta;   // layout r * 3 + k
        float pr = bk[k] + bk[3 + k] * d1[k] + bk[6 + k] * dav[k] + bk[9 + k] * dnv[0] + bk[12 + k] * dnv[1] +
                   bk[15 + k] * dnv[2];
        g.pred[k] = pr;
        gw += gN[k] * pr;
        const float gp = gN[k] * g.w;
        gd1[k] = gp * bk[3 + k];
        gda_[k] = gp * bk[6 + k];
        gdn[0] += gp * bk[9 + k];
        gdn[1] += gp * bk[12 + k];
        gdn[2] += gp * bk[15 + k];
        if (kNeedBeta) {
            g.gbeta[k] = gp;
            g.gbeta[3 + k] = gp * d1[k];
            g.gbeta[6 + k] = gp * dav[k];
            g.gbeta[9 + k] = gp * dnv[0];
            g.gbeta[12 + k] = gp * dnv[1];
            g.gbeta[15 + k] = gp * dnv[2];
        }
    }
    const float gdist = -gw * e;
    const float t = 2.f * gdist * rV;
    g.gdf = make_float3(gd1[0] * rden + t * df[0], gd1[1] * rden + t * df[1], gd1[2] * rden + t * df[2]);
    g.gden = -(gd1[0] * d1[0] + gd1[1] * d1[1] + gd1[2] * d1[2]) * rden;
    g.gV = -gdist * dist * rV;
    g.gda = make_float3(gda_[0], gda_[1], gda_[2]);
    g.gdn = make_float3(gdn[0], gdn[1], gdn[2]);
}

CD_DEV void centre_range(int pos, int n, int hw, int sp, int &lo, int &hi)
{
    lo = max(0, idivup(pos - hw, sp));
    hi = min((n - 1) / sp, (pos + hw) / sp);
}

// ---------------------------------------------------------------------------
// Pass 2: reconstruction backward, pixel side.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) recon_grad_pixel_kernel(GArgs A)
{
    const int ox = blockIdx.x * blockDim.x + threadIdx.x, oy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ox >= A.Wr || oy >= A.Hr) return;
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W, R = (size_t)A.Hr * A.Wr, C = (size_t)A.Hs * A.Ws;
    const int px = ox * A.rs, py = oy * A.rs;
    const size_t p = b * P + (size_t)py * A.W + px, o = b * R + (size_t)oy * A.Wr + ox;
    int sx, ex, sy, ey;
    centre_range(px, A.W, A.hw, A.sp, sx, ex);
    centre_range(py, A.H, A.hw, A.sp, sy, ey);
    const float3 ap = f3(A.alb, p), np_ = f3(A.nrm, p);
    float3 galb = make_float3(0.f, 0.f, 0.f), gnn = galb;
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        const float3 fp = f3(B_.f, p);
        const float vp = __ldg(B_.v + p), sp_ = __ldg(B_.s + p);
        float N[3] = {0.f, 0.f, 0.f}, D = 0.f;
        const float zero[3] = {0.f, 0.f, 0.f};
        PairGrad g;
        for (int iy = sy; iy <= ey; ++iy)
            for (int ix = sx; ix <= ex; ++ix) {
                const size_t c = b * P + (size_t)(iy * A.sp) * A.W + ix * A.sp;
                const float3 fc = f3(B_.f, c), ac = f3(A.alb, c), nc = f3(A.nrm, c);
                const float3 da = make_float3(ap.x - ac.x, ap.y - ac.y, ap.z - ac.z);
                const float3 dn = make_float3(np_.x - nc.x, np_.y - nc.y, np_.z - nc.z);
                recon_pair<false>(fp, fc, sp_, __ldg(B_.s + c), vp, __ldg(B_.v + c), da, dn,
                                  B_.beta + (b * C + (size_t)iy * A.Ws + ix) * kBeta, zero, 0.f, g);
                N[0] += g.w * g.pred[0];
                N[1] += g.w * g.pred[1];
                N[2] += g.w * g.pred[2];
                D += g.w;
            }
        const float Dt = fmaxf(D, 1e-7f);
        const float3 G = f3(B_.gout, o);
        const float Gv[3] = {G.x, G.y, G.z};
        float gN[3], gD = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float ok = N[k] / Dt;
            gN[k] = ok > 0.f ? Gv[k] / Dt : 0.f;
            gD -= gN[k] * ok;
        }
        if (!(D > 1e-7f)) gD = 0.f;
        B_.gN[3 * o] = gN[0];
        B_.gN[3 * o + 1] = gN[1];
        B_.gN[3 * o + 2] = gN[2];
        B_.gD[o] = gD;
        float3 gf = make_float3(0.f, 0.f, 0.f);
        float gs = 0.f, gv = 0.f;
        for (int iy = sy; iy <= ey; ++iy)
            for (int ix = sx; ix <= ex; ++ix) {
                const size_t c = b * P + (size_t)(iy * A.sp) * A.W + ix * A.sp;
                const float3 fc = f3(B_.f, c), ac = f3(A.alb, c), nc = f3(A.nrm, c);
                const float3 da = make_float3(ap.x - ac.x, ap.y - ac.y, ap.z - ac.z);
                const float3 dn = make_float3(np_.x - nc.x, np_.y - nc.y, np_.z - nc.z);
                recon_pair<false>(fp, fc, sp_, __ldg(B_.s + c), vp, __ldg(B_.v + c), da, dn,
                                  B_.beta + (b * C + (size_t)iy * A.Ws + ix) * kBeta, gN, gD, g);
                gf.x += g.gdf.x;
                gf.y += g.gdf.y;
                gf.z += g.gdf.z;
                gs += g.gden;
                gv += g.gV;
                galb.x += g.gda.x;
                galb.y += g.gda.y;
                galb.z += g.gda.z;
                gnn.x += g.gdn.x;
                gnn.y += g.gdn.y;
                gnn.z += g.gdn.z;
            }
        add3(B_.gf, p, gf);
        B_.gs[p] += gs;
        B_.gv[p] += gv;
    }
    add3(A.galb, p, galb);
    add3(A.gn, p, gnn);
}

// Pass 2 with the tile's centres staged in shared memory: a CTA of 32 x 8
// output pixels first copies, for every centre any of its pixels reaches
// (the forward recon kernel's superset), both buffers' features, standard
// deviation, variance and coefficients and the shared albedo and normal into
// one record of kRecG floats; the per-pixel loops then read records instead
// of global memory.  Same pairs, same order, same arithmetic as
// recon_grad_pixel_kernel, so the same results.
constexpr int kRecG = 52;   // fA[3] sA vA betaA[18] | fB[3] sB vB betaB[18] | alb[3] nrm[3]

__host__ __device__ inline int floordiv_g(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

__host__ __device__ inline size_t recon_grad_smem(int hw, int sp, int rs)
{
    const int ncx = (31 * rs + 2 * hw) / sp + 2, ncy = (7 * rs + 2 * hw) / sp + 2;
    return (size_t)ncx * ncy * kRecG * sizeof(float);
}

__global__ void __launch_bounds__(256) recon_grad_pixel_smem_kernel(GArgs A)
{
    extern __shared__ float recs[];
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W, R = (size_t)A.Hr * A.Wr, C = (size_t)A.Hs * A.Ws;
    const int ox0 = blockIdx.x * 32, oy0 = blockIdx.y * 8;
    const int ox1 = min(ox0 + 31, A.Wr - 1), oy1 = min(oy0 + 7, A.Hr - 1);
    const int cx_lo = max(0, floordiv_g(ox0 * A.rs - A.hw, A.sp)), cx_hi = min(A.Ws - 1, (ox1 * A.rs + A.hw) / A.sp);
    const int cy_lo = max(0, floordiv_g(oy0 * A.rs - A.hw, A.sp)), cy_hi = min(A.Hs - 1, (oy1 * A.rs + A.hw) / A.sp);
    const int ncx = cx_hi - cx_lo + 1, ncy = cy_hi - cy_lo + 1;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    // one thread per (centre, field group)
    for (int e = tid; e < ncx * ncy * 4; e += 256) {
        const int n = e >> 2, part = e & 3;
        const int iy = cy_lo + n / ncx, ix = cx_lo + n % ncx;
        const size_t c = b * P + (size_t)(iy * A.sp) * A.W + ix * A.sp;
        const size_t ci = b * C + (size_t)iy * A.Ws + ix;
        float *r = recs + (size_t)n * kRecG;
        if (part < 2) {
            const GBuf &B_ = A.bf[part];
            float *q = r + 23 * part;
            const float3 f = f3(B_.f, c);
            q[0] = f.x;
            q[1] = f.y;
            q[2] = f.z;
            q[3] = __ldg(B_.s + c);
            q[4] = __ldg(B_.v + c);
#pragma unroll
            for (int k = 0; k < 9; ++k) q[5 + k] = __ldg(B_.beta + ci * kBeta + k);
        } else if (part == 2) {
#pragma unroll
            for (int X = 0; X < 2; ++X)
#pragma unroll
                for (int k = 9; k < kBeta; ++k) r[23 * X + 5 + k] = __ldg(A.bf[X].beta + ci * kBeta + k);
        } else {
            const float3 al = f3(A.alb, c), nr = f3(A.nrm, c);
            r[46] = al.x;
            r[47] = al.y;
            r[48] = al.z;
            r[49] = nr.x;
            r[50] = nr.y;
            r[51] = nr.z;
        }
    }
    __syncthreads();

    const int ox = ox0 + threadIdx.x, oy = oy0 + threadIdx.y;
    if (ox >= A.Wr || oy >= A.Hr) return;
    const int px = ox * A.rs, py = oy * A.rs;
    const size_t p = b * P + (size_t)py * A.W + px, o = b * R + (size_t)oy * A.Wr + ox;
    int sx, ex, sy, ey;
    centre_range(px, A.W, A.hw, A.sp, sx, ex);
    centre_range(py, A.H, A.hw, A.sp, sy, ey);
    const float3 ap = f3(A.alb, p), np_ = f3(A.nrm, p);
    float3 galb = make_float3(0.f, 0.f, 0.f), gnn = galb;
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        const float3 fp = f3(B_.f, p);
        const float vp = __ldg(B_.v + p), sp_ = __ldg(B_.s + p);
        float N[3] = {0.f, 0.f, 0.f}, D = 0.f;
        const float zero[3] = {0.f, 0.f, 0.f};
        PairGrad g;
        for (int iy = sy; iy <= ey; ++iy)
            for (int ix = sx; ix <= ex; ++ix) {
                const float *r = recs + (size_t)((iy - cy_lo) * ncx + (ix - cx_lo)) * kRecG;
                const float *q = r + 23 * X;
                const float3 da = make_float3(ap.x - r[46], ap.y - r[47], ap.z - r[48]);
                const float3 dn = make_float3(np_.x - r[49], np_.y - r[50], np_.z - r[51]);
                recon_pair<false>(fp, make_float3(q[0], q[1], q[2]), sp_, q[3], vp, q[4], da, dn, q + 5, zero, 0.f,
                                  g);
                N[0] += g.w * g.pred[0];
                N[1] += g.w * g.pred[1];
                N[2] += g.w * g.pred[2];
                D += g.w;
            }
        const float Dt = fmaxf(D, 1e-7f);
        const float3 G = f3(B_.gout, o);
        const float Gv[3] = {G.x, G.y, G.z};
        float gN[3], gD = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float ok = N[k] / Dt;
            gN[k] = ok > 0.f ? Gv[k] / Dt : 0.f;
            gD -= gN[k] * ok;
        }
        if (!(D > 1e-7f)) gD = 0.f;
        B_.gN[3 * o] = gN[0];
        B_.gN[3 * o + 1] = gN[1];
        B_.gN[3 * o + 2] = gN[2];
        B_.gD[o] = gD;
        float3 gf = make_float3(0.f, 0.f, 0.f);
        float gs = 0.f, gv = 0.f;
        for (int iy = sy; iy <= ey; ++iy)
            for (int ix = sx; ix <= ex; ++ix) {
                const float *r = recs + (size_t)((iy - cy_lo) * ncx + (ix - cx_lo)) * kRecG;
                const float *q = r + 23 * X;
                const float3 da = make_float3(ap.x - r[46], ap.y - r[47], ap.z - r[48]);
                const float3 dn = make_float3(np_.x - r[49], np_.y - r[50], np_.z - r[51]);
                recon_pair<false>(fp, make_float3(q[0], q[1], q[2]), sp_, q[3], vp, q[4], da, dn, q + 5, gN, gD, g);
                gf.x += g.gdf.x;
                gf.y += g.gdf.y;
                gf.z += g.gdf.z;
                gs += g.gden;
                gv += g.gV;
                galb.x += g.gda.x;
                galb.y += g.gda.y;
                galb.z += g.gda.z;
                gnn.x += g.gdn.x;
                gnn.y += g.gdn.y;
                gnn.z += g.gdn.z;
            }
        add3(B_.gf, p, gf);
        B_.gs[p] += gs;
        B_.gv[p] += gv;
    }
    add3(A.galb, p, galb);
    add3(A.gn, p, gnn);
}

// ---------------------------------------------------------------------------
// Pass 3: reconstruction backward, centre side (dL/dbeta and the centre's
// own features).  The output pixels whose centre range contains c are found
// by testing the forward's range rule on a slightly wider candidate set.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) recon_grad_centre_kernel(GArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= A.Ws || j >= A.Hs) return;
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W, R = (size_t)A.Hr * A.Wr, C = (size_t)A.Hs * A.Ws;
    const size_t c = b * P + (size_t)(j * A.sp) * A.W + i * A.sp;
    const size_t ci = b * C + (size_t)j * A.Ws + i;
    const int ox0 = max(0, (i * A.sp - A.hw - A.sp) / A.rs), ox1 = min(A.Wr - 1, (i * A.sp + A.hw + A.sp) / A.rs);
    const int oy0 = max(0, (j * A.sp - A.hw - A.sp) / A.rs), oy1 = min(A.Hr - 1, (j * A.sp + A.hw + A.sp) / A.rs);
    // which candidate output pixels have (i, j) in their centre range, tested
    // once per axis (the range's lower end follows the reference's iDivUp,
    // which is not monotone near the image's top and left edges, so the
    // set need not be an interval); at most 64 candidates per axis are kept
    // as bits, more fall back to testing inside the loop
    const int nxc = ox1 - ox0 + 1, nyc = oy1 - oy0 + 1;
    const bool use_bits = nxc <= 64 && nyc <= 64;
    unsigned long long xbits = 0ull, ybits = 0ull;
    if (use_bits) {
        for (int ox = ox0; ox <= ox1; ++ox) {
            int sx, ex;
            centre_range(ox * A.rs, A.W, A.hw, A.sp, sx, ex);
            if (i >= sx && i <= ex) xbits |= 1ull << (ox - ox0);
        }
        for (int oy = oy0; oy <= oy1; ++oy) {
            int sy, ey;
            centre_range(oy * A.rs, A.H, A.hw, A.sp, sy, ey);
            if (j >= sy && j <= ey) ybits |= 1ull << (oy - oy0);
        }
    }
    auto x_in = [&](int ox) {
        if (use_bits) return ((xbits >> (ox - ox0)) & 1ull) != 0;
        int sx, ex;
        centre_range(ox * A.rs, A.W, A.hw, A.sp, sx, ex);
        return i >= sx && i <= ex;
    };
    auto y_in = [&](int oy) {
        if (use_bits) return ((ybits >> (oy - oy0)) & 1ull) != 0;
        int sy, ey;
        centre_range(oy * A.rs, A.H, A.hw, A.sp, sy, ey);
        return j >= sy && j <= ey;
    };
    const float3 ac = f3(A.alb, c), nc = f3(A.nrm, c);
    float3 galb = make_float3(0.f, 0.f, 0.f), gnn = galb;
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        const float3 fc = f3(B_.f, c);
        const float vc = __ldg(B_.v + c), sc = __ldg(B_.s + c);
        const float *beta = B_.beta + ci * kBeta;
        float gb[kBeta];
#pragma unroll
        for (int k = 0; k < kBeta; ++k) gb[k] = 0.f;
        float3 gf = make_float3(0.f, 0.f, 0.f);
        float gs = 0.f, gv = 0.f;
        PairGrad g;
        for (int oy = oy0; oy <= oy1; ++oy) {
            if (!y_in(oy)) continue;
            for (int ox = ox0; ox <= ox1; ++ox) {
                if (!x_in(ox)) continue;
                const size_t p = b * P + (size_t)(oy * A.rs) * A.W + ox * A.rs;
                const size_t o = b * R + (size_t)oy * A.Wr + ox;
                const float3 ap = f3(A.alb, p), np_ = f3(A.nrm, p);
                const float3 da = make_float3(ap.x - ac.x, ap.y - ac.y, ap.z - ac.z);
                const float3 dn = make_float3(np_.x - nc.x, np_.y - nc.y, np_.z - nc.z);
                const float gN[3] = {B_.gN[3 * o], B_.gN[3 * o + 1], B_.gN[3 * o + 2]};
                recon_pair<true>(f3(B_.f, p), fc, __ldg(B_.s + p), sc, __ldg(B_.v + p), vc, da, dn, beta, gN,
                                 B_.gD[o], g);
#pragma unroll
                for (int k = 0; k < kBeta; ++k) gb[k] += g.gbeta[k];
                gf.x -= g.gdf.x;
                gf.y -= g.gdf.y;
                gf.z -= g.gdf.z;
                gs += g.gden;
                gv += g.gV;
                galb.x -= g.gda.x;
                galb.y -= g.gda.y;
                galb.z -= g.gda.z;
                gnn.x -= g.gdn.x;
                gnn.y -= g.gdn.y;
                gnn.z -= g.gdn.z;
            }
        }
#pragma unroll
        for (int k = 0; k < kBeta; ++k) B_.gbeta[ci * kBeta + k] = gb[k];
        add3(B_.gf, c, gf);
        B_.gs[c] += gs;
        B_.gv[c] += gv;
    }
    add3(A.galb, c, galb);
    add3(A.gn, c, gnn);
}

// One regression tap of one buffer: the forward quantities and the
// derivatives of dL with respect to the tap's inputs, given u and beta.
struct TapGrad {
    float3 gdf, gy, gda, gdn;   // dL/d(f_t - f_c), dL/dy_t, dL/d(alb_t - alb_c), dL/d(n_t - n_c)
    float gden, gV;
};

CD_DEV void regression_tap(float3 ft, float3 fc, float3 yt, float st, float sc, float vt, float vc, float3 da,
                           float3 dn, const float *u, const float *beta, TapGrad &g)
{
    const float df[3] = {ft.x - fc.x, ft.y - fc.y, ft.z - fc.z};
    const float dav[3] = {da.x, da.y, da.z}, dnv[3] = {dn.x, dn.y, dn.z};
    const float yv[3] = {yt.x, yt.y, yt.z};
    const float den = (sc + st) + 1e-2f;
    const float V = (vc + vt) + 1e-4f;
    const float rden = __fdividef(1.f, den), rV = __fdividef(1.f, V);   // as in recon_pair
    const float dist = (df[0] * df[0] + df[1] * df[1] + df[2] * df[2]) * rV;
    const float e = __expf(-dist);
    const float w = e + 1e-7f;
    float gw = 0.f, gd1[3], gda[3], gdn[3] = {0.f, 0.f, 0.f}, d1[3], gyv[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        d1[k] = df[k] * rden;
        const float dl[kP] = {1.f, d1[k], dav[k], dnv[0], dnv[1], dnv[2]};
        float a = 0.f, c = 0.f;
#pragma unroll
        for (int r = 0; r < kP; ++r) {
            a += u[r * 3 + k] * dl[r];
            c += beta[r * 3 + k] * dl[r];
        }
        const float res = yv[k] - c;
        gw += a * res;
        gyv[k] = w * a;
        // dL/ddelta_r = w (u_r res - a beta_r)
        gd1[k] = w * (u[3 + k] * res - a * beta[3 + k]);
        gda[k] = w * (u[6 + k] * res - a * beta[6 + k]);
        gdn[0] += w * (u[9 + k] * res - a * beta[9 + k]);
        gdn[1] += w * (u[12 + k] * res - a * beta[12 + k]);
        gdn[2] += w * (u[15 + k] * res - a * beta[15 + k]);
    }
    const float gdist = -gw * e;
    const float t = 2.f * gdist * rV;
    g.gdf = make_float3(gd1[0] * rden + t * df[0], gd1[1] * rden + t * df[1], gd1[2] * rden + t * df[2]);
    g.gden = -(gd1[0] * d1[0] + gd1[1] * d1[1] + gd1[2] * d1[2]) * rden;
    g.gV = -gdist * dist * rV;
    g.gy = make_float3(gyv[0], gyv[1], gyv[2]);
    g.gda = make_float3(gda[0], gda[1], gda[2]);
    g.gdn = make_float3(gdn[0], gdn[1], gdn[2]);
}

// ---------------------------------------------------------------------------
// Pass 4: u = A^-1 dL/dbeta with the stored Cholesky factor, then the
// centre-side terms of every window tap.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) regression_grad_centre_kernel(GArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= A.Ws || j >= A.Hs) return;
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W, C = (size_t)A.Hs * A.Ws;
    const int cx = i * A.sp, cy = j * A.sp;
    const size_t c = b * P + (size_t)cy * A.W + cx;
    const size_t ci = b * C + (size_t)j * A.Ws + i;
    const float3 ac = f3(A.alb, c), nc = f3(A.nrm, c);
    float3 galb = make_float3(0.f, 0.f, 0.f), gnn = galb;
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        float u[kBeta], beta[kBeta];
#pragma unroll
        for (int k = 0; k < kBeta; ++k) beta[k] = __ldg(B_.beta + ci * kBeta + k);
        // per channel: L z = g, L^T u = z (L lower triangular, row-major packed)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float *Lk = B_.L + ci * kL + 21 * k;
            float z[kP];
#pragma unroll
            for (int r = 0; r < kP; ++r) {
                float s = B_.gbeta[ci * kBeta + r * 3 + k];
#pragma unroll
                for (int q = 0; q < r; ++q) s -= __ldg(Lk + r * (r + 1) / 2 + q) * z[q];
                z[r] = s / __ldg(Lk + r * (r + 1) / 2 + r);
            }
#pragma unroll
            for (int r = kP - 1; r >= 0; --r) {
                float s = z[r];
#pragma unroll
                for (int q = r + 1; q < kP; ++q) s -= __ldg(Lk + q * (q + 1) / 2 + r) * u[q * 3 + k];
                u[r * 3 + k] = s / __ldg(Lk + r * (r + 1) / 2 + r);
            }
        }
#pragma unroll
        for (int k = 0; k < kBeta; ++k) B_.u[ci * kBeta + k] = u[k];
        const float3 fc = f3(B_.f, c);
        const float vc = __ldg(B_.v + c), sc = __ldg(B_.s + c);
        float3 gf = make_float3(0.f, 0.f, 0.f);
        float gs = 0.f, gv = 0.f;
        TapGrad g;
        for (int dy = -A.hw; dy <= A.hw; ++dy) {
            const int ty = mirror(cy + dy, A.H);
            for (int dx = -A.hw; dx <= A.hw; ++dx) {
                const size_t t = b * P + (size_t)ty * A.W + mirror(cx + dx, A.W);
                const float3 at = f3(A.alb, t), nt = f3(A.nrm, t);
                regression_tap(f3(B_.f, t), fc, f3(B_.y, t), __ldg(B_.s + t), sc, __ldg(B_.v + t), vc,
                               make_float3(at.x - ac.x, at.y - ac.y, at.z - ac.z),
                               make_float3(nt.x - nc.x, nt.y - nc.y, nt.z - nc.z), u, beta, g);
                gf.x -= g.gdf.x;
                gf.y -= g.gdf.y;
                gf.z -= g.gdf.z;
                gs += g.gden;
                gv += g.gV;
                galb.x -= g.gda.x;
                galb.y -= g.gda.y;
                galb.z -= g.gda.z;
                gnn.x -= g.gdn.x;
                gnn.y -= g.gdn.y;
                gnn.z -= g.gdn.z;
            }
        }
        add3(B_.gf, c, gf);
        B_.gs[c] += gs;
        B_.gv[c] += gv;
    }
    add3(A.galb, c, galb);
    add3(A.gn, c, gnn);
}

// ---------------------------------------------------------------------------
// Pass 5: tap-side terms gathered per pixel q.  Window position t of
// centre c maps to pixel mirror(t); along each axis the positions whose
// image is q are q itself, -q (q <= hw) and 2n-2-q (the far border).
// ---------------------------------------------------------------------------
CD_DEV int tap_positions(int q, int n, int hw, int cmax, int out[3])
{
    int k = 0;
    out[k++] = q;
    if (q >= 1 && -q >= -hw) out[k++] = -q;
    if (q <= n - 2 && 2 * n - 2 - q <= cmax + hw && 2 * n - 2 - q >= n) out[k++] = 2 * n - 2 - q;
    return k;
}

__global__ void __launch_bounds__(256) regression_grad_tap_kernel(GArgs A)
{
    const int qx = blockIdx.x * blockDim.x + threadIdx.x, qy = blockIdx.y * blockDim.y + threadIdx.y;
    if (qx >= A.W || qy >= A.H) return;
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W, C = (size_t)A.Hs * A.Ws;
    const size_t q = b * P + (size_t)qy * A.W + qx;
    int txs[3], tys[3];
    const int ntx = tap_positions(qx, A.W, A.hw, (A.Ws - 1) * A.sp, txs);
    const int nty = tap_positions(qy, A.H, A.hw, (A.Hs - 1) * A.sp, tys);
    const float3 at = f3(A.alb, q), nt = f3(A.nrm, q);
    float3 galb = make_float3(0.f, 0.f, 0.f), gnn = galb;
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        const float3 ft = f3(B_.f, q), yt = f3(B_.y, q);
        const float vt = __ldg(B_.v + q), st = __ldg(B_.s + q);
        float3 gf = make_float3(0.f, 0.f, 0.f), gy = gf;
        float gs = 0.f, gv = 0.f;
        TapGrad g;
        for (int a = 0; a < nty; ++a) {
            const int ty = tys[a];
            const int j0 = max(0, (ty - A.hw + A.sp - 1) >= 0 ? (ty - A.hw + A.sp - 1) / A.sp : 0);
            const int j1 = min(A.Hs - 1, (ty + A.hw) >= 0 ? (ty + A.hw) / A.sp : -1);
            for (int j = j0; j <= j1; ++j) {
                if (abs(j * A.sp - ty) > A.hw) continue;
                for (int bb = 0; bb < ntx; ++bb) {
                    const int tx = txs[bb];
                    const int i0 = max(0, (tx - A.hw + A.sp - 1) >= 0 ? (tx - A.hw + A.sp - 1) / A.sp : 0);
                    const int i1 = min(A.Ws - 1, (tx + A.hw) >= 0 ? (tx + A.hw) / A.sp : -1);
                    for (int i = i0; i <= i1; ++i) {
                        if (abs(i * A.sp - tx) > A.hw) continue;
                        const size_t c = b * P + (size_t)(j * A.sp) * A.W + i * A.sp;
                        const size_t ci = b * C + (size_t)j * A.Ws + i;
                        const float3 ac = f3(A.alb, c), nc = f3(A.nrm, c);
                        regression_tap(ft, f3(B_.f, c), yt, st, __ldg(B_.s + c), vt, __ldg(B_.v + c),
                                       make_float3(at.x - ac.x, at.y - ac.y, at.z - ac.z),
                                       make_float3(nt.x - nc.x, nt.y - nc.y, nt.z - nc.z), B_.u + ci * kBeta,
                                       B_.beta + ci * kBeta, g);
                        gf.x += g.gdf.x;
                        gf.y += g.gdf.y;
                        gf.z += g.gdf.z;
                        gy.x += g.gy.x;
                        gy.y += g.gy.y;
                        gy.z += g.gy.z;
                        gs += g.gden;
                        gv += g.gV;
                        galb.x += g.gda.x;
                        galb.y += g.gda.y;
                        galb.z += g.gda.z;
                        gnn.x += g.gdn.x;
                        gnn.y += g.gdn.y;
                        gnn.z += g.gdn.z;
                    }
                }
            }
        }
        add3(B_.gf, q, gf);
        add3(B_.gy, q, gy);
        B_.gs[q] += gs;
        B_.gv[q] += gv;
    }
    add3(A.galb, q, galb);
    add3(A.gn, q, gnn);
}

// Pass 5 with the tile's centres staged in shared memory.  Along each axis
// the centres any pixel of a 32 x 8 tile reaches (directly, or through the
// reflect-101 images -q near the low edge and 2n-2-q near the high edge,
// which only occur when the direct range already reaches centre 0 or the
// last centre) form one range [lo, hi]; a record per centre holds both
// buffers' features, standard deviation, variance, u and coefficients and
// the shared albedo and normal.  Same pairs, order and arithmetic as
// regression_grad_tap_kernel.
constexpr int kRecT = 88;   // per buffer X at 41 X: f[3] s v u[18] beta[18]; alb[3] at 82, nrm[3] at 85

__host__ __device__ inline size_t tap_grad_smem(int hw, int sp)
{
    const int ncx = (31 + 2 * hw) / sp + 2, ncy = (7 + 2 * hw) / sp + 2;
    return (size_t)ncx * ncy * kRecT * sizeof(float);
}

__global__ void __launch_bounds__(256) regression_grad_tap_smem_kernel(GArgs A)
{
    extern __shared__ float recs[];
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W, C = (size_t)A.Hs * A.Ws;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 8;
    const int x1 = min(x0 + 31, A.W - 1), y1 = min(y0 + 7, A.H - 1);
    const int cx_lo = x0 - A.hw > 0 ? (x0 - A.hw + A.sp - 1) / A.sp : 0;
    const int cy_lo = y0 - A.hw > 0 ? (y0 - A.hw + A.sp - 1) / A.sp : 0;
    const int cx_hi = min(A.Ws - 1, (x1 + A.hw) / A.sp), cy_hi = min(A.Hs - 1, (y1 + A.hw) / A.sp);
    const int ncx = cx_hi - cx_lo + 1, ncy = cy_hi - cy_lo + 1;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int e = tid; e < ncx * ncy * 5; e += 256) {
        const int n = e / 5, part = e - 5 * n;
        const int iy = cy_lo + n / ncx, ix = cx_lo + n % ncx;
        const size_t c = b * P + (size_t)(iy * A.sp) * A.W + ix * A.sp;
        const size_t ci = b * C + (size_t)iy * A.Ws + ix;
        float *r = recs + (size_t)n * kRecT;
        if (part < 2) {                       // features, sd, var, u of buffer `part`
            const GBuf &B_ = A.bf[part];
            float *q = r + 41 * part;
            const float3 f = f3(B_.f, c);
            q[0] = f.x;
            q[1] = f.y;
            q[2] = f.z;
            q[3] = __ldg(B_.s + c);
            q[4] = __ldg(B_.v + c);
#pragma unroll
            for (int k = 0; k < kBeta; ++k) q[5 + k] = B_.u[ci * kBeta + k];
        } else if (part < 4) {                // coefficients of buffer part - 2
            const GBuf &B_ = A.bf[part - 2];
            float *q = r + 41 * (part - 2) + 23;
#pragma unroll
            for (int k = 0; k < kBeta; ++k) q[k] = __ldg(B_.beta + ci * kBeta + k);
        } else {
            const float3 al = f3(A.alb, c), nr = f3(A.nrm, c);
            r[82] = al.x;
            r[83] = al.y;
            r[84] = al.z;
            r[85] = nr.x;
            r[86] = nr.y;
            r[87] = nr.z;
        }
    }
    __syncthreads();

    const int qx = x0 + threadIdx.x, qy = y0 + threadIdx.y;
    if (qx >= A.W || qy >= A.H) return;
    const size_t q = b * P + (size_t)qy * A.W + qx;
    int txs[3], tys[3];
    const int ntx = tap_positions(qx, A.W, A.hw, (A.Ws - 1) * A.sp, txs);
    const int nty = tap_positions(qy, A.H, A.hw, (A.Hs - 1) * A.sp, tys);
    const float3 at = f3(A.alb, q), nt = f3(A.nrm, q);
    float3 galb = make_float3(0.f, 0.f, 0.f), gnn = galb;
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        const float3 ft = f3(B_.f, q), yt = f3(B_.y, q);
        const float vt = __ldg(B_.v + q), st = __ldg(B_.s + q);
        float3 gf = make_float3(0.f, 0.f, 0.f), gy = gf;
        float gs = 0.f, gv = 0.f;
        TapGrad g;
        for (int a = 0; a < nty; ++a) {
            const int ty = tys[a];
            const int j0 = max(0, (ty - A.hw + A.sp - 1) >= 0 ? (ty - A.hw + A.sp - 1) / A.sp : 0);
            const int j1 = min(A.Hs - 1, (ty + A.hw) >= 0 ? (ty + A.hw) / A.sp : -1);
            for (int j = j0; j <= j1; ++j) {
                if (abs(j * A.sp - ty) > A.hw) continue;
                for (int bb = 0; bb < ntx; ++bb) {
                    const int tx = txs[bb];
                    const int i0 = max(0, (tx - A.hw + A.sp - 1) >= 0 ? (tx - A.hw + A.sp - 1) / A.sp : 0);
                    const int i1 = min(A.Ws - 1, (tx + A.hw) >= 0 ? (tx + A.hw) / A.sp : -1);
                    for (int i = i0; i <= i1; ++i) {
                        if (abs(i * A.sp - tx) > A.hw) continue;
                        const float *r = recs + (size_t)((j - cy_lo) * ncx + (i - cx_lo)) * kRecT;
                        const float *rq = r + 41 * X;
                        regression_tap(ft, make_float3(rq[0], rq[1], rq[2]), yt, st, rq[3], vt, rq[4],
                                       make_float3(at.x - r[82], at.y - r[83], at.z - r[84]),
                                       make_float3(nt.x - r[85], nt.y - r[86], nt.z - r[87]), rq + 5, rq + 23, g);
                        gf.x += g.gdf.x;
                        gf.y += g.gdf.y;
                        gf.z += g.gdf.z;
                        gy.x += g.gy.x;
                        gy.y += g.gy.y;
                        gy.z += g.gy.z;
                        gs += g.gden;
                        gv += g.gV;
                        galb.x += g.gda.x;
                        galb.y += g.gda.y;
                        galb.z += g.gda.z;
                        gnn.x += g.gdn.x;
                        gnn.y += g.gdn.y;
                        gnn.z += g.gdn.z;
                    }
                }
            }
        }
        add3(B_.gf, q, gf);
        add3(B_.gy, q, gy);
        B_.gs[q] += gs;
        B_.gv[q] += gv;
    }
    add3(A.galb, q, galb);
    add3(A.gn, q, gnn);
}

// ---------------------------------------------------------------------------
// Pass 6a: dL/dv (through sqrt, the regression, the reconstruction and the
// variance output) and the variance's own derivative:
// v_p = |m_p - f_p|^2, m_p = mean of the in-bounds neighbours (without p).
// h_p = 2 (m_p - f_p) dL/dv_p: f_p gets -h_p, each neighbour h_p / n_p
// (gathered in pass 6b).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) variance_grad_kernel(GArgs A)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= A.W || y >= A.H) return;
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W;
    const size_t p = b * P + (size_t)y * A.W + x;
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        const float s = __ldg(B_.s + p);
        float gv = B_.gv[p] + (s > 0.f ? B_.gs[p] / (2.f * s) : 0.f);
        if (B_.gvar) gv += __ldg(B_.gvar + p);
        const int sx = max(0, x - 1), ex = min(A.W - 1, x + 1), sy = max(0, y - 1), ey = min(A.H - 1, y + 1);
        float m[3] = {0.f, 0.f, 0.f};
        int n = 0;
        for (int iy = sy; iy <= ey; ++iy)
            for (int ix = sx; ix <= ex; ++ix) {
                if (ix == x && iy == y) continue;
                const float3 v = f3(B_.f, b * P + (size_t)iy * A.W + ix);
                m[0] += v.x;
                m[1] += v.y;
                m[2] += v.z;
                ++n;
            }
        const float3 fp = f3(B_.f, p);
        const float inv = n > 0 ? 1.f / (float)n : 0.f;
        const float h[3] = {2.f * (m[0] * inv - fp.x) * gv, 2.f * (m[1] * inv - fp.y) * gv,
                            2.f * (m[2] * inv - fp.z) * gv};
        B_.hn[3 * p] = h[0] * inv;
        B_.hn[3 * p + 1] = h[1] * inv;
        B_.hn[3 * p + 2] = h[2] * inv;
        add3(B_.gf, p, make_float3(-h[0], -h[1], -h[2]));
    }
}

// Pass 6b: neighbours' variance terms and the assembly:
// dL/dimga = gf(A) + gy(B), dL/dimgb = gf(B) + gy(A).
__global__ void __launch_bounds__(256) assemble_grad_kernel(GArgs A)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= A.W || y >= A.H) return;
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W;
    const size_t p = b * P + (size_t)y * A.W + x;
    float3 g[2];
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        float3 v = f3(B_.gf, p);
        for (int iy = max(0, y - 1); iy <= min(A.H - 1, y + 1); ++iy)
            for (int ix = max(0, x - 1); ix <= min(A.W - 1, x + 1); ++ix) {
                if (ix == x && iy == y) continue;
                const float3 h = f3(B_.hn, b * P + (size_t)iy * A.W + ix);
                v.x += h.x;
                v.y += h.y;
                v.z += h.z;
            }
        g[X] = v;
    }
    const float3 ya = f3(A.bf[0].gy, p), yb = f3(A.bf[1].gy, p);
    st3(A.out_a, p, make_float3(g[0].x + yb.x, g[0].y + yb.y, g[0].z + yb.z));
    st3(A.out_b, p, make_float3(g[1].x + ya.x, g[1].y + ya.y, g[1].z + ya.z));
    st3(A.out_alb, p, f3(A.galb, p));
    st3(A.out_n, p, f3(A.gn, p));
}

}  // namespace

size_t regression_grad_workspace_floats(int B, int H, int W, int sp, int rs)
{
    const size_t P = (size_t)B * H * W, R = (size_t)B * (H / rs) * (W / rs), C = (size_t)B * (H / sp) * (W / sp);
    // per buffer: v, s, gf(3), gy(3), gs, gv, hn(3) = 13 P; beta, L, u, gbeta = 117 C; gN(3), gD = 4 R
    // shared: galb(3), gn(3) = 6 P
    return 2 * (13 * P + 117 * C + 4 * R) + 6 * P;
}

// The workspace begins with the forward's quantities, in this order:
// variance and standard deviation of A, then of B (P floats each), the
// coefficients [buf][C][18] and the Cholesky factors [buf][C][63].
cudaError_t launch_regression_keep(const float *imga, const float *imgb, const float *albedo, const float *normal,
                                   float *outa, float *outb, float *vara, float *varb, int B, int H, int W, int win,
                                   int sp, int rs, float *ws, cudaStream_t st)
{
    const size_t P = (size_t)B * H * W, C = (size_t)B * (H / sp) * (W / sp);
    float *v0 = ws, *s0 = ws + P, *v1 = ws + 2 * P, *s1 = ws + 3 * P;
    float *beta = ws + 4 * P, *L = beta + 2 * C * kBeta;
    cudaError_t e;
    if ((e = launch_variance(imga, imgb, v0, v1, s0, s1, B, H, W, st)) != cudaSuccess) return e;
    if ((e = launch_regression(imga, imgb, albedo, normal, v0, v1, s0, s1, beta, B, H, W, win, sp, st, L)) !=
        cudaSuccess)
        return e;
    if ((e = launch_recon(imga, imgb, albedo, normal, v0, v1, s0, s1, beta, outa, outb, B, H, W, win, sp, rs, st)) !=
        cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(vara, v0, P * sizeof(float), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    return cudaMemcpyAsync(varb, v1, P * sizeof(float), cudaMemcpyDeviceToDevice, st);
}

cudaError_t launch_regression_grad(const float *imga, const float *imgb, const float *albedo, const float *normal,
                                   const float *g_outa, const float *g_outb, const float *g_vara,
                                   const float *g_varb, float *g_imga, float *g_imgb, float *g_albedo,
                                   float *g_normal, int B, int H, int W, int win, int sp, int rs, float *ws,
                                   cudaStream_t st, bool kept)
{
    const size_t P = (size_t)B * H * W, R = (size_t)B * (H / rs) * (W / rs), C = (size_t)B * (H / sp) * (W / sp);
    GArgs A{};
    A.H = H;
    A.W = W;
    A.hw = win / 2;
    A.sp = sp;
    A.rs = rs;
    A.Hs = H / sp;
    A.Ws = W / sp;
    A.Hr = H / rs;
    A.Wr = W / rs;
    float *cur = ws;
    auto take = [&](size_t n) {
        float *p = cur;
        cur += n;
        return p;
    };
    float *var[2], *sd[2], *beta, *L, *u[2], *gbeta[2];
    for (int X = 0; X < 2; ++X) {
        var[X] = take(P);
        sd[X] = take(P);
    }
    beta = take(2 * C * kBeta);   // [buf][C][18], the layout the forward kernels use
    L = take(2 * C * kL);
    for (int X = 0; X < 2; ++X) {
        u[X] = take(C * kBeta);
        gbeta[X] = take(C * kBeta);
    }
    float *zero_begin = cur;      // everything below is accumulated and starts at zero
    for (int X = 0; X < 2; ++X) {
        GBuf &g = A.bf[X];
        g.f = X ? imgb : imga;
        g.y = X ? imga : imgb;
        g.v = var[X];
        g.s = sd[X];
        g.beta = beta + X * C * kBeta;
        g.L = L + X * C * kL;
        g.u = u[X];
        g.gbeta = gbeta[X];
        g.gN = take(3 * R);
        g.gD = take(R);
        g.gf = take(3 * P);
        g.gy = take(3 * P);
        g.gs = take(P);
        g.gv = take(P);
        g.hn = take(3 * P);
        g.gout = X ? g_outb : g_outa;
        g.gvar = X ? g_varb : g_vara;
    }
    A.alb = albedo;
    A.nrm = normal;
    A.galb = take(3 * P);
    A.gn = take(3 * P);
    A.out_a = g_imga;
    A.out_b = g_imgb;
    A.out_alb = g_albedo;
    A.out_n = g_normal;
    cudaError_t e = cudaMemsetAsync(zero_begin, 0, (size_t)(cur - zero_begin) * sizeof(float), st);
    if (e != cudaSuccess) return e;

    // pass 1: forward quantities (variance, std, coefficients, Cholesky
    // factors), unless launch_regression_keep left them in the workspace
    if (!kept) {
        if ((e = launch_variance(imga, imgb, var[0], var[1], sd[0], sd[1], B, H, W, st)) != cudaSuccess) return e;
        if ((e = launch_regression(imga, imgb, albedo, normal, var[0], var[1], sd[0], sd[1], beta, B, H, W, win,
                                   sp, st, L)) != cudaSuccess)
            return e;
    }
    dim3 blk(32, 8);
    dim3 g_out((A.Wr + 31) / 32, (A.Hr + 7) / 8, B), g_cen((A.Ws + 31) / 32, (A.Hs + 7) / 8, B);
    dim3 g_px((W + 31) / 32, (H + 7) / 8, B);
    const size_t rg_smem = recon_grad_smem(A.hw, A.sp, A.rs);
    if (rg_smem <= 200 * 1024) {
        if ((e = cudaFuncSetAttribute(recon_grad_pixel_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)rg_smem)) != cudaSuccess)
            return e;
        recon_grad_pixel_smem_kernel<<<g_out, blk, rg_smem, st>>>(A);
    } else {
        recon_grad_pixel_kernel<<<g_out, blk, 0, st>>>(A);
    }
    recon_grad_centre_kernel<<<g_cen, blk, 0, st>>>(A);
    regression_grad_centre_kernel<<<dim3((A.Ws + 15) / 16, (A.Hs + 7) / 8, B), dim3(16, 8), 0, st>>>(A);
    const size_t tg_smem = tap_grad_smem(A.hw, A.sp);
    if (tg_smem <= 200 * 1024) {
        if ((e = cudaFuncSetAttribute(regression_grad_tap_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)tg_smem)) != cudaSuccess)
            return e;
        regression_grad_tap_smem_kernel<<<g_px, blk, tg_smem, st>>>(A);
    } else {
        regression_grad_tap_kernel<<<g_px, blk, 0, st>>>(A);
    }
    variance_grad_kernel<<<g_px, blk, 0, st>>>(A);
    assemble_grad_kernel<<<g_px, blk, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace cd
