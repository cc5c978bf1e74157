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
//   1. variance + std, forward regression keeping each centre's Cholesky factor,
//      reconstruction keeping each output pixel's outputs and weight sum D
//   2. recon backward, pixel side (dL/dN, dL/dD from the kept outputs and D,
//      stored per output pixel)
//   3. recon backward, centre side (dL/dbeta), one thread per (centre,
//      buffer), the output rows streamed through shared memory
//   4. solve backward (u) and the regression's centre-side terms, one thread
//      per (centre, buffer), the window rows streamed through shared memory
//   5. the regression's tap-side terms, gathered per pixel over every
//      (centre, window position) whose reflect-101 image is that pixel
//   6. sqrt / variance chain and assembly of dL/dimga, dL/dimgb, dL/dalbedo,
//      dL/dnormal.
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "f32x2.cuh"
#include "window_rows.cuh"

namespace cd {
namespace {

constexpr int kP = 6, kBeta = 18, kL = 63;

struct GBuf {
    const float *f, *y, *v, *s, *beta, *L;
    float *u, *gbeta, *gN, *gD, *gf, *gs, *gv, *hn;
    float *gt, *gvs;   // the tap side's own planes: dL/d(image X), and its variance term
    const float *gout, *gvar;   // upstream dL/dout [R,3], dL/dvar [P] (nullable)
};

struct GArgs {
    GBuf bf[2];
    const float4 *state;        // forward recon: (out[3], D) per [buffer][output pixel]
    float4 *crec;               // per centre: head and coefficient pairs, kRecG2 float4s
    float4 *upair;              // per centre: u pairs by channel, 9 float4s
    const float *alb, *nrm;
    float *galb, *gn, *galb_t, *gn_t;
    float *out_a, *out_b, *out_alb, *out_n;   // final gradients
    int B, H, W, hw, sp, rs, Hs, Ws, Hr, Wr;
    bool u_rows;   // pass 4 also writes u as [buffer][centre][18] (for the unstaged tap pass)
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

// dL/dN and dL/dD of one output pixel, from the forward's outputs and weight
// sum (out_k = max(0, N_k / max(D, 1e-7))): dL/dN_k = dL/dout_k / max(D, 1e-7)
// where out_k > 0, else 0; dL/dD = -sum_k dL/dN_k out_k, 0 where D <= 1e-7.
CD_DEV void recon_upstream(float4 S, float3 G, float gN[3], float &gD)
{
    const float Dt = fmaxf(S.w, 1e-7f);
    const float ov[3] = {S.x, S.y, S.z}, Gv[3] = {G.x, G.y, G.z};
    gD = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        gN[k] = ov[k] > 0.f ? Gv[k] / Dt : 0.f;
        gD -= gN[k] * ov[k];
    }
    if (!(S.w > 1e-7f)) gD = 0.f;
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
        PairGrad g;
        float gN[3], gD;
        recon_upstream(A.state[X * (size_t)gridDim.z * R + o], f3(B_.gout, o), gN, gD);
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

// Pass 2 with the tile's centres staged in shared memory and both buffers
// of a pair evaluated as packed FP32x2 lanes (low A, high B).  A CTA of
// 32 x 8 output pixels first copies, for every centre any of its pixels
// reaches (the forward recon kernel's superset), one record of kRecG2
// float4s (pairs (A, B) unless noted):
//   0  f.x f.y   1  f.z s   2  v | alb.x alb.y (scalars)   3  alb.z nrm.xyz (scalars)
//   4 + 3k + m   coefficients of channel k, rows 2m and 2m + 1
// A warp covers 4 x 8 pixels of the tile, so its lanes step through the
// same or neighbouring records (shared-memory broadcast).
constexpr int kRecG2 = 13;

__host__ __device__ inline int floordiv_g(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

__host__ __device__ inline size_t recon_grad_smem(int hw, int sp, int rs)
{
    const int ncx = (31 * rs + 2 * hw) / sp + 2, ncy = (7 * rs + 2 * hw) / sp + 2;
    return (size_t)ncx * ncy * kRecG2 * sizeof(float4);
}

CD_DEV x2::f2 neg2(x2::f2 v) { return v ^ 0x8000000080000000ull; }
CD_DEV x2::f2 dup2(float v) { return x2::pack(v, v); }
CD_DEV x2::f2 rcp2(x2::f2 v) { return x2::pack(__fdividef(1.f, x2::lo(v)), __fdividef(1.f, x2::hi(v))); }
CD_DEV x2::f2 expneg2(x2::f2 v) { return x2::pack(__expf(-x2::lo(v)), __expf(-x2::hi(v))); }

// A tile's centres [cx_lo, cx_lo + ncx) x [cy_lo, cy_lo + ncy) of image b.
struct CentreTile {
    int b, x0, y0, cx_lo, cy_lo, ncx, ncy;
};

CD_DEV void cp_async16(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// The centre records of the pixel- and tap-side passes, built once per
// backward in their shared-memory layout (kRecG2 float4s per centre: the
// head, then the coefficient pairs of channel k, rows 2m and 2m + 1, at
// 4 + 3k + m), so that a tile stages them with 16-byte copies.
__global__ void __launch_bounds__(256) centre_records_kernel(GArgs A)
{
    const size_t C = (size_t)A.B * A.Hs * A.Ws, P = (size_t)A.H * A.W;
    const size_t idx = (size_t)blockIdx.x * 256 + threadIdx.x;
    if (idx >= C * kRecG2) return;
    const size_t ci = idx / kRecG2;
    const int j = (int)(idx - ci * kRecG2);
    const int per = A.Hs * A.Ws, b = (int)(ci / per), r = (int)(ci - (size_t)b * per);
    const int iy = r / A.Ws, ix = r - iy * A.Ws;
    const size_t c = b * P + (size_t)(iy * A.sp) * A.W + ix * A.sp;
    float4 v;
    if (j == 0) {
        v = make_float4(__ldg(A.bf[0].f + 3 * c), __ldg(A.bf[1].f + 3 * c), __ldg(A.bf[0].f + 3 * c + 1),
                        __ldg(A.bf[1].f + 3 * c + 1));
    } else if (j == 1) {
        v = make_float4(__ldg(A.bf[0].f + 3 * c + 2), __ldg(A.bf[1].f + 3 * c + 2), __ldg(A.bf[0].s + c),
                        __ldg(A.bf[1].s + c));
    } else if (j == 2) {
        v = make_float4(__ldg(A.bf[0].v + c), __ldg(A.bf[1].v + c), __ldg(A.alb + 3 * c), __ldg(A.alb + 3 * c + 1));
    } else if (j == 3) {
        v = make_float4(__ldg(A.alb + 3 * c + 2), __ldg(A.nrm + 3 * c), __ldg(A.nrm + 3 * c + 1),
                        __ldg(A.nrm + 3 * c + 2));
    } else {
        const int k = (j - 4) / 3, m = (j - 4) - 3 * k;
        const float *pa = A.bf[0].beta + ci * kBeta, *pb = A.bf[1].beta + ci * kBeta;
        v = make_float4(__ldg(pa + 6 * m + k), __ldg(pb + 6 * m + k), __ldg(pa + 6 * m + 3 + k),
                        __ldg(pb + 6 * m + 3 + k));
    }
    A.crec[idx] = v;
}

// Copy (cp.async, 16 bytes each) the NQ float4s per centre of src for a
// tile's centres into rec, record n at rec + n * stride + off.
template <int NQ>
CD_DEV void stage_records(float4 *rec, int stride, int off, const float4 *src, const GArgs &A, const CentreTile &T,
                          int tid)
{
    const size_t C = (size_t)A.Hs * A.Ws;
    const int nrec = T.ncx * T.ncy;
    const float rncx = 1.f / (float)T.ncx;
    for (int e = tid; e < nrec * NQ; e += 256) {
        const int n = e / NQ, j = e - n * NQ;
        const int ry = (int)(((float)n + 0.5f) * rncx), rx = n - ry * T.ncx;
        const size_t ci = T.b * C + (size_t)(T.cy_lo + ry) * A.Ws + T.cx_lo + rx;
        cp_async16(rec + (size_t)n * stride + off + j, src + ci * NQ + j);
    }
}

CD_DEV CentreTile pixel_tile(const GArgs &A, int t, int tx, int ty)
{
    CentreTile T;
    T.b = t / (tx * ty);
    const int r = t - T.b * tx * ty, by = r / tx, bx = r - by * tx;
    T.x0 = bx * 32;
    T.y0 = by * 8;
    const int ox1 = min(T.x0 + 31, A.Wr - 1), oy1 = min(T.y0 + 7, A.Hr - 1);
    T.cx_lo = max(0, floordiv_g(T.x0 * A.rs - A.hw, A.sp));
    T.cy_lo = max(0, floordiv_g(T.y0 * A.rs - A.hw, A.sp));
    T.ncx = min(A.Ws - 1, (ox1 * A.rs + A.hw) / A.sp) - T.cx_lo + 1;
    T.ncy = min(A.Hs - 1, (oy1 * A.rs + A.hw) / A.sp) - T.cy_lo + 1;
    return T;
}

// The per-pixel inputs of the pixel side, loaded one tile ahead.
struct PixIn2 {
    float3 ap, np, fa, fb, goa, gob;
    float sa, sb, va, vb;
    float4 sta, stb;
};

CD_DEV void load_pixel_x2(const GArgs &A, const CentreTile &T, int warp, int lane, PixIn2 &I)
{
    const size_t P = (size_t)A.H * A.W, R = (size_t)A.Hr * A.Wr;
    const int ox = T.x0 + 4 * warp + (lane & 3), oy = T.y0 + (lane >> 2);
    if (ox >= A.Wr || oy >= A.Hr) return;
    const size_t p = T.b * P + (size_t)(oy * A.rs) * A.W + ox * A.rs, o = T.b * R + (size_t)oy * A.Wr + ox;
    I.ap = f3(A.alb, p);
    I.np = f3(A.nrm, p);
    I.fa = f3(A.bf[0].f, p);
    I.fb = f3(A.bf[1].f, p);
    I.sa = __ldg(A.bf[0].s + p);
    I.sb = __ldg(A.bf[1].s + p);
    I.va = __ldg(A.bf[0].v + p);
    I.vb = __ldg(A.bf[1].v + p);
    I.sta = A.state[o];
    I.stb = A.state[(size_t)A.B * R + o];
    I.goa = f3(A.bf[0].gout, o);
    I.gob = f3(A.bf[1].gout, o);
}

// the pixel side of one output pixel of tile T (warp covers 4 x 8 pixels)
CD_DEV void recon_grad_pixel_x2(const GArgs &A, const CentreTile &T, const float4 *rec4, int warp, int lane,
                                const PixIn2 &I)
{
    using namespace x2;
    const size_t P = (size_t)A.H * A.W, R = (size_t)A.Hr * A.Wr;
    const int ox = T.x0 + 4 * warp + (lane & 3), oy = T.y0 + (lane >> 2);
    if (ox >= A.Wr || oy >= A.Hr) return;
    const int px = ox * A.rs, py = oy * A.rs;
    const size_t p = T.b * P + (size_t)py * A.W + px, o = T.b * R + (size_t)oy * A.Wr + ox;
    int sx, ex, sy, ey;
    centre_range(px, A.W, A.hw, A.sp, sx, ex);
    centre_range(py, A.H, A.hw, A.sp, sy, ey);
    const float3 ap = I.ap, np_ = I.np;
    const f2 fp0 = pack(I.fa.x, I.fb.x), fp1 = pack(I.fa.y, I.fb.y), fp2 = pack(I.fa.z, I.fb.z);
    const f2 spp = pack(I.sa, I.sb), vpp = pack(I.va, I.vb);
    // dL/dN and dL/dD of the pixel, both buffers
    f2 gN0, gN1, gN2, gD;
    {
        float na[3], nb[3], da, db;
        recon_upstream(I.sta, I.goa, na, da);
        recon_upstream(I.stb, I.gob, nb, db);
        for (int X = 0; X < 2; ++X) {
            const float *g = X ? nb : na;
            A.bf[X].gN[3 * o] = g[0];
            A.bf[X].gN[3 * o + 1] = g[1];
            A.bf[X].gN[3 * o + 2] = g[2];
            A.bf[X].gD[o] = X ? db : da;
        }
        gN0 = pack(na[0], nb[0]);
        gN1 = pack(na[1], nb[1]);
        gN2 = pack(na[2], nb[2]);
        gD = pack(da, db);
    }
    const f2 k1e2 = pack(1e-2f, 1e-2f), k1e4 = pack(1e-4f, 1e-4f), k1e7 = pack(1e-7f, 1e-7f);
    const f2 two = pack(2.f, 2.f);
    f2 gf0 = 0ull, gf1 = 0ull, gf2 = 0ull, gs = 0ull, gv = 0ull;
    f2 ga0 = 0ull, ga1 = 0ull, ga2 = 0ull, gn0 = 0ull, gn1 = 0ull, gn2 = 0ull;
    for (int iy = sy; iy <= ey; ++iy)
        for (int ix = sx; ix <= ex; ++ix) {
            const float4 *R4 = rec4 + (size_t)((iy - T.cy_lo) * T.ncx + (ix - T.cx_lo)) * kRecG2;
            const ulonglong2 *RR = reinterpret_cast<const ulonglong2 *>(R4);
            const ulonglong2 h0 = RR[0], h1 = RR[1];
            const float4 q2 = R4[2], q3 = R4[3];
            const f2 df0 = sub2(fp0, h0.x), df1 = sub2(fp1, h0.y), df2 = sub2(fp2, h1.x);
            const f2 rden = rcp2(add2(add2(spp, h1.y), k1e2));
            const f2 rV = rcp2(add2(add2(vpp, pack(q2.x, q2.y)), k1e4));
            const f2 dist = mul2(sqnorm2(df0, df1, df2), rV);
            const f2 e = expneg2(dist);
            const f2 w = add2(e, k1e7);
            const f2 da[3] = {dup2(ap.x - q2.z), dup2(ap.y - q2.w), dup2(ap.z - q3.x)};
            const f2 dn0 = dup2(np_.x - q3.y), dn1 = dup2(np_.y - q3.z), dn2 = dup2(np_.z - q3.w);
            const f2 df[3] = {df0, df1, df2}, gN[3] = {gN0, gN1, gN2};
            f2 gw = gD, gsum = 0ull;
            f2 gd1[3], d1[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const ulonglong2 b01 = RR[4 + 3 * k], b23 = RR[5 + 3 * k], b45 = RR[6 + 3 * k];
                d1[k] = mul2(df[k], rden);
                const f2 pr = fma2(b45.y, dn2, fma2(b45.x, dn1, fma2(b23.y, dn0,
                                   fma2(b23.x, da[k], fma2(b01.y, d1[k], b01.x)))));
                gw = fma2(gN[k], pr, gw);
                const f2 gp = mul2(gN[k], w);
                gd1[k] = mul2(gp, b01.y);
                gsum = fma2(gd1[k], d1[k], gsum);
                if (k == 0) ga0 = fma2(gp, b23.x, ga0);
                if (k == 1) ga1 = fma2(gp, b23.x, ga1);
                if (k == 2) ga2 = fma2(gp, b23.x, ga2);
                gn0 = fma2(gp, b23.y, gn0);
                gn1 = fma2(gp, b45.x, gn1);
                gn2 = fma2(gp, b45.y, gn2);
            }
            const f2 gdist = neg2(mul2(gw, e));
            const f2 t = mul2(mul2(two, gdist), rV);
            gf0 = add2(gf0, fma2(t, df0, mul2(gd1[0], rden)));
            gf1 = add2(gf1, fma2(t, df1, mul2(gd1[1], rden)));
            gf2 = add2(gf2, fma2(t, df2, mul2(gd1[2], rden)));
            gs = sub2(gs, mul2(gsum, rden));
            gv = sub2(gv, mul2(mul2(gdist, dist), rV));
        }
    for (int X = 0; X < 2; ++X) {
        const GBuf &B_ = A.bf[X];
        // the first writer of these planes (zeroed before the passes): a
        // store, without the read of an accumulate
        const float x0 = X ? hi(gf0) : lo(gf0), x1 = X ? hi(gf1) : lo(gf1), x2_ = X ? hi(gf2) : lo(gf2);
        st3(B_.gf, p, make_float3(x0, x1, x2_));
        B_.gs[p] = X ? hi(gs) : lo(gs);
        B_.gv[p] = X ? hi(gv) : lo(gv);
    }
    st3(A.galb, p, make_float3(lo(ga0) + hi(ga0), lo(ga1) + hi(ga1), lo(ga2) + hi(ga2)));
    st3(A.gn, p, make_float3(lo(gn0) + hi(gn0), lo(gn1) + hi(gn1), lo(gn2) + hi(gn2)));
}

// Persistent: a CTA takes tiles t, t + grid, ...; the next tile's records are
// copied (cp.async) into the second buffer while the current tile computes.
__global__ void __launch_bounds__(256, 2) recon_grad_pixel_x2_kernel(GArgs A, int tx, int ty, int ntiles, int cap)
{
    extern __shared__ float4 rec4[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, G = gridDim.x;
    auto stage = [&](int t, int s) {
        const CentreTile T = pixel_tile(A, t, tx, ty);
        stage_records<kRecG2>(rec4 + (size_t)s * cap, kRecG2, 0, A.crec, A, T, threadIdx.x);
    };
    PixIn2 I;
    if ((int)blockIdx.x < ntiles) {
        stage(blockIdx.x, 0);
        load_pixel_x2(A, pixel_tile(A, blockIdx.x, tx, ty), warp, lane, I);
    }
    cp_async_commit();
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += G, ++it) {
        if (t + G < ntiles) stage(t + G, (it + 1) & 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        recon_grad_pixel_x2(A, pixel_tile(A, t, tx, ty), rec4 + (size_t)(it & 1) * cap, warp, lane, I);
        // the next tile's pixel inputs, in flight across the barrier and the staging
        if (t + G < ntiles) load_pixel_x2(A, pixel_tile(A, t + G, tx, ty), warp, lane, I);
        __syncthreads();
    }
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
// Pass 3: reconstruction backward, centre side (dL/dbeta and the centre's
// own features).  Built like pass 4: a CTA owns 32 consecutive centres of one
// centre row, warp 0 takes buffer A and warp 1 buffer B, one thread per
// (centre, buffer).  The output rows whose centre range holds the centre row
// stream through two shared-memory row slots (cp.async, double buffered); a
// slot stores, per output pixel of the row segment the 32 centres' candidate
// columns cover, six float4 groups: g0..g3 as the regression's window rows
// (window_rows.cuh), g4 = (dL/dN_A.xyz, dL/dD_A), g5 = (dL/dN_B.xyz, dL/dD_B),
// positions de-interleaved by the centre spacing sp / rs when rs divides sp
// (32 lanes then read 32 consecutive float4s).  Each thread tests the
// forward's range rule once per candidate column (bits; the rule's lower
// end follows the reference's iDivUp, which is not monotone near the image's
// top and left edges, so the set need not be an interval), and the CTA steps
// through the span of its lanes' columns.
// ---------------------------------------------------------------------------
struct RconGeom {
    int nc;     // candidate columns (and rows) per centre
    int st;     // de-interleave stride: sp / rs when rs divides sp, else 1
    int rw;     // row segment width in output pixels
    int q;      // positions per de-interleaved run
    int npos;   // positions per group (q * st)
};

__host__ __device__ inline RconGeom rcon_geom(int hw, int sp, int rs)
{
    RconGeom g;
    g.nc = (2 * (hw + sp)) / rs + 2;
    g.st = sp % rs == 0 ? sp / rs : 1;
    g.rw = ((kRowCentres - 1) * sp) / rs + g.nc + 1;
    g.q = (g.rw + g.st - 1) / g.st;
    g.npos = g.q * g.st;
    return g;
}

__host__ __device__ inline size_t recon_centre_smem(int hw, int sp, int rs)
{
    const RconGeom g = rcon_geom(hw, sp, rs);
    return (size_t)2 * 6 * g.npos * sizeof(float4) + (size_t)2 * g.rw * sizeof(int) + 64 * sizeof(int) +
           (size_t)kRowCentres * 6 * sizeof(float);
}

__host__ __device__ inline bool recon_centre_rows_ok(int hw, int sp, int rs)
{
    return rcon_geom(hw, sp, rs).nc <= 64 && recon_centre_smem(hw, sp, rs) <= 200 * 1024;
}

__global__ void __launch_bounds__(64, 7) recon_grad_centre_rows_kernel(GArgs A)
{
    extern __shared__ float4 sm4[];
    const RconGeom g = rcon_geom(A.hw, A.sp, A.rs);
    const int slot = 6 * g.npos;   // float4s per slot
    int *pos_ox = reinterpret_cast<int *>(sm4 + 2 * slot);
    int *pos_dst = pos_ox + g.rw;
    int *rows = pos_dst + g.rw;
    float *other = reinterpret_cast<float *>(rows + 64);   // buffer B's albedo / normal terms
    __shared__ int nrows_s;
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W, R = (size_t)A.Hr * A.Wr, C = (size_t)A.Hs * A.Ws;
    const int i0 = blockIdx.x * kRowCentres, j = blockIdx.y;
    const int X = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int seg = floordiv_g(i0 * A.sp - A.hw - A.sp, A.rs);   // output column of position 0

    for (int p = threadIdx.x; p < g.rw; p += 64) {
        pos_ox[p] = clampi(seg + p, 0, A.Wr - 1);
        pos_dst[p] = (p % g.st) * g.q + p / g.st;
    }
    if (threadIdx.x == 0) {
        // output rows whose centre range holds centre row j, in order
        const int oy0 = floordiv_g(j * A.sp - A.hw - A.sp, A.rs);
        int n = 0;
        for (int t = 0; t < g.nc; ++t) {
            const int oy = oy0 + t;
            if (oy < 0 || oy >= A.Hr) continue;
            int sy, ey;
            centre_range(oy * A.rs, A.H, A.hw, A.sp, sy, ey);
            if (j >= sy && j <= ey) rows[n++] = oy;
        }
        nrows_s = n;
    }
    __syncthreads();
    const int nrows = nrows_s;

    const float *imga = A.bf[0].f + 3 * P * b, *imgb = A.bf[1].f + 3 * P * b;
    const float *alb = A.alb + 3 * P * b, *nrm = A.nrm + 3 * P * b;
    const float *vara = A.bf[0].v + P * b, *varb = A.bf[1].v + P * b;
    const float *sda = A.bf[0].s + P * b, *sdb = A.bf[1].s + P * b;
    const float *gNa = A.bf[0].gN + 3 * R * b, *gNb = A.bf[1].gN + 3 * R * b;
    const float *gDa = A.bf[0].gD + R * b, *gDb = A.bf[1].gD + R * b;
    auto stage = [&](int k, int s) {
        const int oy = rows[k];
        float *base = reinterpret_cast<float *>(sm4 + s * slot);
        const size_t prow = (size_t)(oy * A.rs) * A.W, orow = (size_t)oy * A.Wr;
        for (int p = threadIdx.x; p < g.rw; p += 64) {
            const int ox = pos_ox[p];
            const size_t q = prow + (size_t)ox * A.rs, o = orow + ox;
            float *d0 = base + 4 * pos_dst[p];
            float *d1 = d0 + 4 * g.npos, *d2 = d0 + 8 * g.npos, *d3 = d0 + 12 * g.npos;
            float *d4 = d0 + 16 * g.npos, *d5 = d0 + 20 * g.npos;
            const float *a = imga + 3 * q, *c = imgb + 3 * q, *l = alb + 3 * q, *n = nrm + 3 * q;
            cp_async4(d0, a); cp_async4(d0 + 1, a + 1); cp_async4(d0 + 2, a + 2); cp_async4(d0 + 3, vara + q);
            cp_async4(d1, c); cp_async4(d1 + 1, c + 1); cp_async4(d1 + 2, c + 2); cp_async4(d1 + 3, varb + q);
            cp_async4(d2, l); cp_async4(d2 + 1, l + 1); cp_async4(d2 + 2, l + 2); cp_async4(d2 + 3, sda + q);
            cp_async4(d3, n); cp_async4(d3 + 1, n + 1); cp_async4(d3 + 2, n + 2); cp_async4(d3 + 3, sdb + q);
            cp_async4(d4, gNa + 3 * o); cp_async4(d4 + 1, gNa + 3 * o + 1); cp_async4(d4 + 2, gNa + 3 * o + 2);
            cp_async4(d4 + 3, gDa + o);
            cp_async4(d5, gNb + 3 * o); cp_async4(d5 + 1, gNb + 3 * o + 1); cp_async4(d5 + 2, gNb + 3 * o + 2);
            cp_async4(d5 + 3, gDb + o);
        }
    };
    if (nrows > 0) stage(0, 0);
    cp_async_commit();

    // the thread's centre (clamped for lanes past the last centre), its
    // candidate columns [cs, cs + nc) and which of them have it in range
    const int i = min(i0 + lane, A.Ws - 1);
    const size_t c = (size_t)(j * A.sp) * A.W + (size_t)i * A.sp;   // within the image
    const size_t ci = b * C + (size_t)j * A.Ws + i;
    const int cs = floordiv_g(i * A.sp - A.hw - A.sp, A.rs);
    unsigned long long xb = 0ull;
    for (int t = 0; t < g.nc; ++t) {
        const int ox = cs + t;
        if (ox < 0 || ox >= A.Wr) continue;
        int sx, ex;
        centre_range(ox * A.rs, A.W, A.hw, A.sp, sx, ex);
        if (i >= sx && i <= ex) xb |= 1ull << t;
    }
    const bool valid = i0 + lane < A.Ws;
    if (!valid) xb = 0ull;
    const unsigned lo_any = __reduce_or_sync(0xffffffffu, (unsigned)xb);
    const unsigned hi_any = __reduce_or_sync(0xffffffffu, (unsigned)(xb >> 32));
    const unsigned long long any = ((unsigned long long)hi_any << 32) | lo_any;
    const int t_lo = any ? __ffsll((long long)any) - 1 : 0, t_hi = any ? 63 - __clzll((long long)any) : -1;
    const int loff = A.sp % A.rs == 0 ? lane : cs - seg;   // the lane's position offset, as de-interleaved

    const float *betap = (X ? A.bf[1].beta : A.bf[0].beta) + ci * kBeta;
    float beta[kBeta], gb[kBeta];
#pragma unroll
    for (int k = 0; k < kBeta; ++k) {
        beta[k] = __ldg(betap + k);
        gb[k] = 0.f;
    }
    const float3 fc = ld3(X ? imgb : imga, c), ac = ld3(alb, c), nc = ld3(nrm, c);
    const float vc = __ldg((X ? varb : vara) + c), sc = __ldg((X ? sdb : sda) + c);
    float3 gf = make_float3(0.f, 0.f, 0.f), galb = gf, gnn = gf;
    float gs = 0.f, gv = 0.f;
    PairGrad pg;
    for (int k = 0; k < nrows; ++k) {
        if (k + 1 < nrows) {
            stage(k + 1, (k + 1) & 1);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float4 *Pp = sm4 + (k & 1) * slot;
        const float4 *Gf = Pp + X * g.npos, *Ga = Pp + 2 * g.npos, *Gn = Pp + 3 * g.npos;
        const float4 *Gg = Pp + (4 + X) * g.npos;
        int tm = t_lo % g.st, td = t_lo / g.st;
        for (int t = t_lo; t <= t_hi; ++t) {
            if ((xb >> t) & 1ull) {
                const int o = tm * g.q + td + loff;
                const float4 f4 = Gf[o], a4 = Ga[o], n4 = Gn[o], g4 = Gg[o];
                const float spx = X ? n4.w : a4.w;   // sdA rides in g2.w, sdB in g3.w
                const float gN[3] = {g4.x, g4.y, g4.z};
                recon_pair<true>(make_float3(f4.x, f4.y, f4.z), fc, spx, sc, f4.w, vc,
                                 make_float3(a4.x - ac.x, a4.y - ac.y, a4.z - ac.z),
                                 make_float3(n4.x - nc.x, n4.y - nc.y, n4.z - nc.z), beta, gN, g4.w, pg);
#pragma unroll
                for (int q = 0; q < kBeta; ++q) gb[q] += pg.gbeta[q];
                gf.x -= pg.gdf.x;
                gf.y -= pg.gdf.y;
                gf.z -= pg.gdf.z;
                gs += pg.gden;
                gv += pg.gV;
                galb.x -= pg.gda.x;
                galb.y -= pg.gda.y;
                galb.z -= pg.gda.z;
                gnn.x -= pg.gdn.x;
                gnn.y -= pg.gdn.y;
                gnn.z -= pg.gdn.z;
            }
            if (++tm == g.st) {
                tm = 0;
                ++td;
            }
        }
        __syncthreads();
    }
    const size_t cp = b * P + c;
    if (valid) {
        const GBuf &B_ = X ? A.bf[1] : A.bf[0];
#pragma unroll
        for (int q = 0; q < kBeta; ++q) B_.gbeta[ci * kBeta + q] = gb[q];
        add3(B_.gf, cp, gf);
        B_.gs[cp] += gs;
        B_.gv[cp] += gv;
    }
    if (X == 1) {
        other[6 * lane] = galb.x;
        other[6 * lane + 1] = galb.y;
        other[6 * lane + 2] = galb.z;
        other[6 * lane + 3] = gnn.x;
        other[6 * lane + 4] = gnn.y;
        other[6 * lane + 5] = gnn.z;
    }
    __syncthreads();
    if (X == 0 && valid) {
        add3(A.galb, cp, make_float3(galb.x + other[6 * lane], galb.y + other[6 * lane + 1],
                                     galb.z + other[6 * lane + 2]));
        add3(A.gn, cp, make_float3(gnn.x + other[6 * lane + 3], gnn.y + other[6 * lane + 4],
                                   gnn.z + other[6 * lane + 5]));
    }
}

// ---------------------------------------------------------------------------
// Pass 4: u = A^-1 dL/dbeta with the stored Cholesky factor, then the
// centre-side terms of every window tap.  Built like the forward regression
// kernel: a CTA owns 32 consecutive centres of one centre row, warp 0 takes
// buffer A and warp 1 buffer B, one thread per (centre, buffer), and the
// window rows stream through two shared-memory row slots (window_rows.cuh;
// cp.async, double buffered), a tap being four conflict-free LDS.128.  The
// albedo and normal terms of a centre's two buffers are summed by warp 0
// (buffer A's terms first) through shared memory.
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t grad_centre_smem(int hw, int sp)
{
    const RowGeom g = row_geom(hw, sp);
    return (size_t)2 * 4 * g.npos * sizeof(float4) + (size_t)2 * g.rw * sizeof(int) +
           (size_t)kRowCentres * 6 * sizeof(float);
}

__global__ void __launch_bounds__(64, 8) regression_grad_centre_kernel(GArgs A)
{
    extern __shared__ float4 sm4[];
    const RowGeom g = row_geom(A.hw, A.sp);
    const int slot = 4 * g.npos;   // float4s per slot
    int *pos_gx = reinterpret_cast<int *>(sm4 + 2 * slot);
    int *pos_dst = pos_gx + g.rw;
    float *other = reinterpret_cast<float *>(pos_dst + g.rw);   // buffer B's albedo / normal terms
    const int b = blockIdx.z;
    const size_t P = (size_t)A.H * A.W, C = (size_t)A.Hs * A.Ws;
    const int i0 = blockIdx.x * kRowCentres, cy = blockIdx.y * A.sp;
    const int X = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int Rw = 2 * A.hw + 1;
    const float *imga = A.bf[0].f + 3 * P * b, *imgb = A.bf[1].f + 3 * P * b;
    const float *alb = A.alb + 3 * P * b, *nrm = A.nrm + 3 * P * b;
    const float *vara = A.bf[0].v + P * b, *varb = A.bf[1].v + P * b;
    const float *sda = A.bf[0].s + P * b, *sdb = A.bf[1].s + P * b;

    row_positions(pos_gx, pos_dst, g, i0 * A.sp - A.hw, A.W, A.sp, threadIdx.x, 64);
    __syncthreads();
    auto stage = [&](int r, int s) {
        stage_window_row(reinterpret_cast<float *>(sm4 + s * slot), g, pos_gx, pos_dst,
                         clampi(mirror(cy - A.hw + r, A.H), 0, A.H - 1), A.W, imga, imgb, alb, nrm, vara, varb, sda,
                         sdb, threadIdx.x, 64);
    };
    stage(0, 0);
    cp_async_commit();

    // the thread's centre (clamped for lanes past the last centre) and u
    const int i = min(i0 + lane, A.Ws - 1);
    const size_t c = (size_t)cy * A.W + (size_t)i * A.sp;   // within the image
    const size_t ci = b * C + (size_t)blockIdx.y * A.Ws + i;
    const float *Lc = (X ? A.bf[1].L : A.bf[0].L) + ci * kL;
    const float *gbeta = (X ? A.bf[1].gbeta : A.bf[0].gbeta) + ci * kBeta;
    const float *betap = (X ? A.bf[1].beta : A.bf[0].beta) + ci * kBeta;
    float u[kBeta], beta[kBeta];
#pragma unroll
    for (int k = 0; k < kBeta; ++k) beta[k] = __ldg(betap + k);
    // per channel: L z = g, L^T u = z (L lower triangular, row-major packed)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float *Lk = Lc + 21 * k;
        float z[kP];
#pragma unroll
        for (int r = 0; r < kP; ++r) {
            float s = gbeta[r * 3 + k];
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
    const bool valid = i0 + lane < A.Ws;
    if (valid) {
        float *up = reinterpret_cast<float *>(A.upair + ci * 9);   // pairs: channel k, row r at 12k + 4(r/2) + 2(r%2)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int r = 0; r < kP; ++r) up[12 * k + 4 * (r >> 1) + 2 * (r & 1) + X] = u[r * 3 + k];
        if (A.u_rows) {
            float *ug = (X ? A.bf[1].u : A.bf[0].u) + ci * kBeta;
#pragma unroll
            for (int k = 0; k < kBeta; ++k) ug[k] = u[k];
        }
    }
    const float3 fc = ld3(X ? imgb : imga, c), ac = ld3(alb, c), nc = ld3(nrm, c);
    const float vc = __ldg((X ? varb : vara) + c), sc = __ldg((X ? sdb : sda) + c);
    const int gfi = X ? 1 : 0, gyi = X ? 0 : 1;   // own features + variance, target

    float3 gf = make_float3(0.f, 0.f, 0.f), galb = gf, gnn = gf;
    float gs = 0.f, gv = 0.f;
    TapGrad tg;
    for (int r = 0; r < Rw; ++r) {
        if (r + 1 < Rw) {
            stage(r + 1, (r + 1) & 1);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float4 *Pp = sm4 + (r & 1) * slot;
        const float4 *Gf = Pp + gfi * g.npos, *Gy = Pp + gyi * g.npos;
        const float4 *Ga = Pp + 2 * g.npos, *Gn = Pp + 3 * g.npos;
        int tm = 0, td = 0;
        for (int t = 0; t < Rw; ++t) {
            const int o = tm * g.q + td + lane;
            const float4 f4 = Gf[o], y4 = Gy[o], a4 = Ga[o], n4 = Gn[o];
            const float st = X ? n4.w : a4.w;   // sdA rides in g2.w, sdB in g3.w
            regression_tap(make_float3(f4.x, f4.y, f4.z), fc, make_float3(y4.x, y4.y, y4.z), st, sc, f4.w, vc,
                           make_float3(a4.x - ac.x, a4.y - ac.y, a4.z - ac.z),
                           make_float3(n4.x - nc.x, n4.y - nc.y, n4.z - nc.z), u, beta, tg);
            gf.x -= tg.gdf.x;
            gf.y -= tg.gdf.y;
            gf.z -= tg.gdf.z;
            gs += tg.gden;
            gv += tg.gV;
            galb.x -= tg.gda.x;
            galb.y -= tg.gda.y;
            galb.z -= tg.gda.z;
            gnn.x -= tg.gdn.x;
            gnn.y -= tg.gdn.y;
            gnn.z -= tg.gdn.z;
            if (++tm == A.sp) {
                tm = 0;
                ++td;
            }
        }
        __syncthreads();
    }
    const size_t cp = b * P + c;
    if (valid) {
        const GBuf &B_ = X ? A.bf[1] : A.bf[0];
        add3(B_.gf, cp, gf);
        B_.gs[cp] += gs;
        B_.gv[cp] += gv;
    }
    if (X == 1) {
        other[6 * lane] = galb.x;
        other[6 * lane + 1] = galb.y;
        other[6 * lane + 2] = galb.z;
        other[6 * lane + 3] = gnn.x;
        other[6 * lane + 4] = gnn.y;
        other[6 * lane + 5] = gnn.z;
    }
    __syncthreads();
    if (X == 0 && valid) {
        add3(A.galb, cp, make_float3(galb.x + other[6 * lane], galb.y + other[6 * lane + 1],
                                     galb.z + other[6 * lane + 2]));
        add3(A.gn, cp, make_float3(gnn.x + other[6 * lane + 3], gnn.y + other[6 * lane + 4],
                                   gnn.z + other[6 * lane + 5]));
    }
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
    float3 galb = make_float3(0.f, 0.f, 0.f), gnn = galb, gfX[2], gyX[2];
    float gvsX[2];
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
        gfX[X] = gf;
        gyX[X] = gy;
        gvsX[X] = gv + (st > 0.f ? gs / (2.f * st) : 0.f);
    }
    // the only writer of its planes: stores
    st3(A.bf[0].gt, q, make_float3(gfX[0].x + gyX[1].x, gfX[0].y + gyX[1].y, gfX[0].z + gyX[1].z));
    st3(A.bf[1].gt, q, make_float3(gfX[1].x + gyX[0].x, gfX[1].y + gyX[0].y, gfX[1].z + gyX[0].z));
    A.bf[0].gvs[q] = gvsX[0];
    A.bf[1].gvs[q] = gvsX[1];
    st3(A.galb_t, q, galb);
    st3(A.gn_t, q, gnn);
}

// Pass 5 with the tile's centres staged in shared memory and both buffers
// as packed FP32x2 lanes.  Along each axis the centres any pixel of a
// 32 x 8 tile reaches (directly, or through the reflect-101 images -q near
// the low edge and 2n-2-q near the high edge, which only occur when the
// direct range already reaches centre 0 or the last centre) form one range
// [lo, hi]; a record of kRecT2 float4s per centre holds (pairs (A, B)
// unless noted):
//   0  f.x f.y   1  f.z s   2  v | alb.x alb.y (scalars)   3  alb.z nrm.xyz (scalars)
//   4 + 3k + m   coefficients of channel k, rows 2m and 2m + 1
//   13 + 3k + m  u of channel k, rows 2m and 2m + 1
// (the first 13 the pixel side's record).  A warp covers 4 x 8 pixels of the
// tile (shared-memory broadcast, as in pass 2).  Same pairs and order as regression_grad_tap_kernel.
constexpr int kRecT2 = 22;

__host__ __device__ inline size_t tap_grad_smem(int hw, int sp)
{
    const int ncx = (31 + 2 * hw) / sp + 2, ncy = (7 + 2 * hw) / sp + 2;
    return (size_t)ncx * ncy * kRecT2 * sizeof(float4);
}

CD_DEV CentreTile tap_tile(const GArgs &A, int t, int tx, int ty)
{
    CentreTile T;
    T.b = t / (tx * ty);
    const int r = t - T.b * tx * ty, by = r / tx, bx = r - by * tx;
    T.x0 = bx * 32;
    T.y0 = by * 8;
    const int x1 = min(T.x0 + 31, A.W - 1), y1 = min(T.y0 + 7, A.H - 1);
    T.cx_lo = T.x0 - A.hw > 0 ? (T.x0 - A.hw + A.sp - 1) / A.sp : 0;
    T.cy_lo = T.y0 - A.hw > 0 ? (T.y0 - A.hw + A.sp - 1) / A.sp : 0;
    T.ncx = min(A.Ws - 1, (x1 + A.hw) / A.sp) - T.cx_lo + 1;
    T.ncy = min(A.Hs - 1, (y1 + A.hw) / A.sp) - T.cy_lo + 1;
    return T;
}

// The per-pixel inputs of the tap side, loaded one tile ahead.
struct PixIn5 {
    float3 at, nt, fa, fb;
    float sa, sb, va, vb;
};

CD_DEV void load_pixel_tap(const GArgs &A, const CentreTile &T, int warp, int lane, PixIn5 &I)
{
    const size_t P = (size_t)A.H * A.W;
    const int qx = T.x0 + 4 * warp + (lane & 3), qy = T.y0 + (lane >> 2);
    if (qx >= A.W || qy >= A.H) return;
    const size_t q = T.b * P + (size_t)qy * A.W + qx;
    I.at = f3(A.alb, q);
    I.nt = f3(A.nrm, q);
    I.fa = f3(A.bf[0].f, q);
    I.fb = f3(A.bf[1].f, q);
    I.sa = __ldg(A.bf[0].s + q);
    I.sb = __ldg(A.bf[1].s + q);
    I.va = __ldg(A.bf[0].v + q);
    I.vb = __ldg(A.bf[1].v + q);
}

// the tap side of one pixel of tile T (warp covers 4 x 8 pixels)
CD_DEV void regression_grad_tap_x2(const GArgs &A, const CentreTile &T, const float4 *rec4, int warp, int lane,
                                   const PixIn5 &I)
{
    using namespace x2;
    const size_t P = (size_t)A.H * A.W;
    const int qx = T.x0 + 4 * warp + (lane & 3), qy = T.y0 + (lane >> 2);
    if (qx >= A.W || qy >= A.H) return;
    const size_t q = T.b * P + (size_t)qy * A.W + qx;
    int txs[3], tys[3];
    const int ntx = tap_positions(qx, A.W, A.hw, (A.Ws - 1) * A.sp, txs);
    const int nty = tap_positions(qy, A.H, A.hw, (A.Hs - 1) * A.sp, tys);
    const float3 at = I.at, nt = I.nt, fqa = I.fa, fqb = I.fb;
    const f2 ft[3] = {pack(fqa.x, fqb.x), pack(fqa.y, fqb.y), pack(fqa.z, fqb.z)};
    const f2 yt[3] = {pack(fqb.x, fqa.x), pack(fqb.y, fqa.y), pack(fqb.z, fqa.z)};   // y of A is imgb
    const f2 stt = pack(I.sa, I.sb), vtt = pack(I.va, I.vb);
    const f2 k1e2 = pack(1e-2f, 1e-2f), k1e4 = pack(1e-4f, 1e-4f), k1e7 = pack(1e-7f, 1e-7f);
    const f2 two = pack(2.f, 2.f);
    f2 gf[3] = {0ull, 0ull, 0ull}, gy[3] = {0ull, 0ull, 0ull}, ga[3] = {0ull, 0ull, 0ull};
    f2 gn0 = 0ull, gn1 = 0ull, gn2 = 0ull, gs = 0ull, gv = 0ull;
    for (int a_ = 0; a_ < nty; ++a_) {
        const int ty = tys[a_];
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
                    const float4 *R4 = rec4 + (size_t)((j - T.cy_lo) * T.ncx + (i - T.cx_lo)) * kRecT2;
                    const ulonglong2 *RR = reinterpret_cast<const ulonglong2 *>(R4);
                    const ulonglong2 h0 = RR[0], h1 = RR[1];
                    const float4 q2 = R4[2], q3 = R4[3];
                    const f2 df[3] = {sub2(ft[0], h0.x), sub2(ft[1], h0.y), sub2(ft[2], h1.x)};
                    const f2 rden = rcp2(add2(add2(h1.y, stt), k1e2));
                    const f2 rV = rcp2(add2(add2(pack(q2.x, q2.y), vtt), k1e4));
                    const f2 dist = mul2(sqnorm2(df[0], df[1], df[2]), rV);
                    const f2 e = expneg2(dist);
                    const f2 w = add2(e, k1e7);
                    const f2 da[3] = {dup2(at.x - q2.z), dup2(at.y - q2.w), dup2(at.z - q3.x)};
                    const f2 dn0 = dup2(nt.x - q3.y), dn1 = dup2(nt.y - q3.z), dn2 = dup2(nt.z - q3.w);
                    f2 gw = 0ull, gsum = 0ull, t1[3], t2[3], d1[3];
                    f2 tn0 = 0ull, tn1 = 0ull, tn2 = 0ull;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const ulonglong2 b01 = RR[4 + 3 * k], b23 = RR[5 + 3 * k], b45 = RR[6 + 3 * k];
                        const ulonglong2 u01 = RR[13 + 3 * k], u23 = RR[14 + 3 * k], u45 = RR[15 + 3 * k];
                        d1[k] = mul2(df[k], rden);
                        const f2 a = fma2(u45.y, dn2, fma2(u45.x, dn1, fma2(u23.y, dn0,
                                         fma2(u23.x, da[k], fma2(u01.y, d1[k], u01.x)))));
                        const f2 c = fma2(b45.y, dn2, fma2(b45.x, dn1, fma2(b23.y, dn0,
                                         fma2(b23.x, da[k], fma2(b01.y, d1[k], b01.x)))));
                        const f2 res = sub2(yt[k], c);
                        gw = fma2(a, res, gw);
                        gy[k] = fma2(w, a, gy[k]);
                        const f2 na = neg2(a);
                        // dL/ddelta_r / w = u_r res - a beta_r
                        t1[k] = fma2(na, b01.y, mul2(u01.y, res));
                        t2[k] = fma2(na, b23.x, mul2(u23.x, res));
                        tn0 = fma2(na, b23.y, fma2(u23.y, res, tn0));
                        tn1 = fma2(na, b45.x, fma2(u45.x, res, tn1));
                        tn2 = fma2(na, b45.y, fma2(u45.y, res, tn2));
                    }
                    const f2 gdist = neg2(mul2(gw, e));
                    const f2 t = mul2(mul2(two, gdist), rV);
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const f2 g1 = mul2(w, t1[k]);
                        gf[k] = add2(gf[k], fma2(t, df[k], mul2(g1, rden)));
                        gsum = fma2(g1, d1[k], gsum);
                        ga[k] = fma2(w, t2[k], ga[k]);
                    }
                    gn0 = fma2(w, tn0, gn0);
                    gn1 = fma2(w, tn1, gn1);
                    gn2 = fma2(w, tn2, gn2);
                    gs = sub2(gs, mul2(gsum, rden));
                    gv = sub2(gv, mul2(mul2(gdist, dist), rV));
                }
            }
        }
    }
    // the only writer of its planes: stores (image A's features are buffer
    // A's and buffer B's target, and the other way round)
    st3(A.bf[0].gt, q, make_float3(lo(gf[0]) + hi(gy[0]), lo(gf[1]) + hi(gy[1]), lo(gf[2]) + hi(gy[2])));
    st3(A.bf[1].gt, q, make_float3(hi(gf[0]) + lo(gy[0]), hi(gf[1]) + lo(gy[1]), hi(gf[2]) + lo(gy[2])));
    A.bf[0].gvs[q] = lo(gv) + (I.sa > 0.f ? lo(gs) / (2.f * I.sa) : 0.f);
    A.bf[1].gvs[q] = hi(gv) + (I.sb > 0.f ? hi(gs) / (2.f * I.sb) : 0.f);
    st3(A.galb_t, q, make_float3(lo(ga[0]) + hi(ga[0]), lo(ga[1]) + hi(ga[1]), lo(ga[2]) + hi(ga[2])));
    st3(A.gn_t, q, make_float3(lo(gn0) + hi(gn0), lo(gn1) + hi(gn1), lo(gn2) + hi(gn2)));
}

// Persistent, the next tile's records copied while the current one computes
// (as recon_grad_pixel_x2_kernel).
__global__ void __launch_bounds__(256, 2) regression_grad_tap_x2_kernel(GArgs A, int tx, int ty, int ntiles, int cap)
{
    extern __shared__ float4 rec4[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, G = gridDim.x;
    auto stage = [&](int t, int s) {
        const CentreTile T = tap_tile(A, t, tx, ty);
        stage_records<kRecG2>(rec4 + (size_t)s * cap, kRecT2, 0, A.crec, A, T, threadIdx.x);
        stage_records<9>(rec4 + (size_t)s * cap, kRecT2, kRecG2, A.upair, A, T, threadIdx.x);
    };
    PixIn5 I;
    if ((int)blockIdx.x < ntiles) {
        stage(blockIdx.x, 0);
        load_pixel_tap(A, tap_tile(A, blockIdx.x, tx, ty), warp, lane, I);
    }
    cp_async_commit();
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += G, ++it) {
        if (t + G < ntiles) stage(t + G, (it + 1) & 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        regression_grad_tap_x2(A, tap_tile(A, t, tx, ty), rec4 + (size_t)(it & 1) * cap, warp, lane, I);
        if (t + G < ntiles) load_pixel_tap(A, tap_tile(A, t + G, tx, ty), warp, lane, I);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Pass 6a: dL/dv (through sqrt, the regression, the reconstruction and the
// variance output) and the variance's own derivative:
// v_p = |m_p - f_p|^2, m_p = mean of the in-bounds neighbours (without p).
// h_p = 2 (m_p - f_p) dL/dv_p: f_p gets -h_p = -n_p (h_p / n_p), each
// neighbour h_p / n_p (both gathered in pass 6b).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) variance_grad_kernel(GArgs A)
{
    // one thread per (pixel, buffer): grid z = image * 2 + buffer
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= A.W || y >= A.H) return;
    const int b = blockIdx.z >> 1, X = blockIdx.z & 1;
    const size_t P = (size_t)A.H * A.W;
    const size_t p = b * P + (size_t)y * A.W + x;
    {
        const GBuf &B_ = X ? A.bf[1] : A.bf[0];
        const float s = __ldg(B_.s + p);
        float gv = B_.gv[p] + (s > 0.f ? B_.gs[p] / (2.f * s) : 0.f) + B_.gvs[p];
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
        // h / n only: the assembly takes f_p's own term as n (h / n), except
        // for a pixel without neighbours (a 1 x 1 image), whose -h goes here
        B_.hn[3 * p] = h[0] * inv;
        B_.hn[3 * p + 1] = h[1] * inv;
        B_.hn[3 * p + 2] = h[2] * inv;
        if (n == 0) add3(B_.gf, p, make_float3(-h[0], -h[1], -h[2]));
    }
}

// Pass 6b: neighbours' variance terms and the assembly with the tap side's
// planes: dL/dimga = gf(A) + gt(A), dL/dimgb = gf(B) + gt(B).
__global__ void __launch_bounds__(256) assemble_grad_kernel(GArgs A)
{
    // one thread per (pixel, image): grid z = batch image * 2 + X; X = 0
    // writes dL/dimga and dL/dalbedo, X = 1 dL/dimgb and dL/dnormal
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= A.W || y >= A.H) return;
    const int b = blockIdx.z >> 1, X = blockIdx.z & 1;
    const size_t P = (size_t)A.H * A.W;
    const size_t p = b * P + (size_t)y * A.W + x;
    const GBuf &B_ = X ? A.bf[1] : A.bf[0];
    const int sx = max(0, x - 1), ex = min(A.W - 1, x + 1), sy = max(0, y - 1), ey = min(A.H - 1, y + 1);
    const float n = (float)((ex - sx + 1) * (ey - sy + 1) - 1);
    const float3 g = f3(B_.gf, p), hp = f3(B_.hn, p);
    float3 v = make_float3(g.x - n * hp.x, g.y - n * hp.y, g.z - n * hp.z);   // f_p's own term -h_p
    for (int iy = sy; iy <= ey; ++iy)
        for (int ix = sx; ix <= ex; ++ix) {
            if (ix == x && iy == y) continue;
            const float3 h = f3(B_.hn, b * P + (size_t)iy * A.W + ix);
            v.x += h.x;
            v.y += h.y;
            v.z += h.z;
        }
    const float3 t = f3(B_.gt, p);
    st3(X ? A.out_b : A.out_a, p, make_float3(v.x + t.x, v.y + t.y, v.z + t.z));
    const float3 c = f3(X ? A.gn : A.galb, p), ct = f3(X ? A.gn_t : A.galb_t, p);
    st3(X ? A.out_n : A.out_alb, p, make_float3(c.x + ct.x, c.y + ct.y, c.z + ct.z));
}

// Workspace layout, offsets in floats, every region 16-byte aligned.  It
// begins with the forward's quantities (kept by launch_regression_keep):
// variance and standard deviation of A, then of B (P floats each), the
// coefficients [buf][C][18], the Cholesky factors [buf][C][63] and the
// reconstruction's (out[3], D) [buf][R] as float4; then the backward's own
// planes, those that are accumulated last and zeroed before the passes.
struct GradLayout {
    size_t var[2], sd[2], beta, L, state, crec, upair, u[2], gbeta[2], gN[2], gD[2], gt[2], gvs[2], hn[2];
    size_t galb_t, gn_t;
    size_t zero_begin, gf[2], gs[2], gv[2], galb, gn, total;
};

GradLayout grad_layout(int B, int H, int W, int sp, int rs)
{
    const size_t P = (size_t)B * H * W, R = (size_t)B * (H / rs) * (W / rs), C = (size_t)B * (H / sp) * (W / sp);
    GradLayout g{};
    size_t cur = 0;
    auto take = [&](size_t n) {
        const size_t at = cur;
        cur += (n + 3) & ~(size_t)3;
        return at;
    };
    for (int X = 0; X < 2; ++X) {
        g.var[X] = take(P);
        g.sd[X] = take(P);
    }
    g.beta = take(2 * C * kBeta);   // [buf][C][18], the layout the forward kernels use
    g.L = take(2 * C * kL);
    g.state = take(2 * R * 4);
    g.crec = take(C * 4 * kRecG2);
    g.upair = take(C * 36);
    for (int X = 0; X < 2; ++X) {
        g.u[X] = take(C * kBeta);
        g.gbeta[X] = take(C * kBeta);
        g.gN[X] = take(3 * R);
        g.gD[X] = take(R);
        g.gt[X] = take(3 * P);
        g.gvs[X] = take(P);
        g.hn[X] = take(3 * P);
    }
    g.galb_t = take(3 * P);
    g.gn_t = take(3 * P);
    g.zero_begin = cur;
    for (int X = 0; X < 2; ++X) {
        g.gf[X] = take(3 * P);
        g.gs[X] = take(P);
        g.gv[X] = take(P);
    }
    g.galb = take(3 * P);
    g.gn = take(3 * P);
    g.total = cur;
    return g;
}

}  // namespace

size_t regression_grad_workspace_floats(int B, int H, int W, int sp, int rs)
{
    return grad_layout(B, H, W, sp, rs).total;
}

cudaError_t launch_regression_keep(const float *imga, const float *imgb, const float *albedo, const float *normal,
                                   float *outa, float *outb, float *vara, float *varb, int B, int H, int W, int win,
                                   int sp, int rs, float *ws, cudaStream_t st)
{
    const GradLayout g = grad_layout(B, H, W, sp, rs);
    const size_t P = (size_t)B * H * W;
    float *v0 = ws + g.var[0], *s0 = ws + g.sd[0], *v1 = ws + g.var[1], *s1 = ws + g.sd[1];
    cudaError_t e;
    if ((e = launch_variance(imga, imgb, v0, v1, s0, s1, B, H, W, st)) != cudaSuccess) return e;
    if ((e = launch_regression(imga, imgb, albedo, normal, v0, v1, s0, s1, ws + g.beta, B, H, W, win, sp, st,
                               ws + g.L)) != cudaSuccess)
        return e;
    if ((e = launch_recon(imga, imgb, albedo, normal, v0, v1, s0, s1, ws + g.beta, outa, outb, B, H, W, win, sp, rs,
                          st, ws + g.state)) != cudaSuccess)
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
    const GradLayout L = grad_layout(B, H, W, sp, rs);
    GArgs A{};
    A.B = B;
    A.H = H;
    A.W = W;
    A.hw = win / 2;
    A.sp = sp;
    A.rs = rs;
    A.Hs = H / sp;
    A.Ws = W / sp;
    A.Hr = H / rs;
    A.Wr = W / rs;
    const size_t C = (size_t)B * A.Hs * A.Ws;
    for (int X = 0; X < 2; ++X) {
        GBuf &g = A.bf[X];
        g.f = X ? imgb : imga;
        g.y = X ? imga : imgb;
        g.v = ws + L.var[X];
        g.s = ws + L.sd[X];
        g.beta = ws + L.beta + X * C * kBeta;
        g.L = ws + L.L + X * C * kL;
        g.u = ws + L.u[X];
        g.gbeta = ws + L.gbeta[X];
        g.gN = ws + L.gN[X];
        g.gD = ws + L.gD[X];
        g.gf = ws + L.gf[X];
        g.gt = ws + L.gt[X];
        g.gvs = ws + L.gvs[X];
        g.gs = ws + L.gs[X];
        g.gv = ws + L.gv[X];
        g.hn = ws + L.hn[X];
        g.gout = X ? g_outb : g_outa;
        g.gvar = X ? g_varb : g_vara;
    }
    A.state = reinterpret_cast<const float4 *>(ws + L.state);
    A.crec = reinterpret_cast<float4 *>(ws + L.crec);
    A.upair = reinterpret_cast<float4 *>(ws + L.upair);
    A.alb = albedo;
    A.nrm = normal;
    A.galb = ws + L.galb;
    A.galb_t = ws + L.galb_t;
    A.gn_t = ws + L.gn_t;
    A.gn = ws + L.gn;
    A.out_a = g_imga;
    A.out_b = g_imgb;
    A.out_alb = g_albedo;
    A.out_n = g_normal;
    // the accumulated planes start at zero, unless the packed pixel side
    // stores every pixel of them first (recon_scale 1)
    const size_t rg_smem = recon_grad_smem(A.hw, A.sp, A.rs), tg_smem = tap_grad_smem(A.hw, A.sp);
    const bool pixel_x2 = 2 * rg_smem <= 200 * 1024, tap_x2 = 2 * tg_smem <= 200 * 1024;
    A.u_rows = !tap_x2;
    cudaError_t e;
    if (!(pixel_x2 && rs == 1) &&
        (e = cudaMemsetAsync(ws + L.zero_begin, 0, (L.total - L.zero_begin) * sizeof(float), st)) != cudaSuccess)
        return e;

    // pass 1: forward quantities (variance, std, coefficients, Cholesky
    // factors, the reconstruction's outputs and weight sums), unless
    // launch_regression_keep left them in the workspace
    if (!kept) {
        float *v0 = ws + L.var[0], *v1 = ws + L.var[1], *s0 = ws + L.sd[0], *s1 = ws + L.sd[1];
        if ((e = launch_variance(imga, imgb, v0, v1, s0, s1, B, H, W, st)) != cudaSuccess) return e;
        if ((e = launch_regression(imga, imgb, albedo, normal, v0, v1, s0, s1, ws + L.beta, B, H, W, win, sp, st,
                                   ws + L.L)) != cudaSuccess)
            return e;
        if ((e = launch_recon(imga, imgb, albedo, normal, v0, v1, s0, s1, ws + L.beta, nullptr, nullptr, B, H, W,
                              win, sp, rs, st, ws + L.state)) != cudaSuccess)
            return e;
    }
    dim3 blk(32, 8);
    dim3 g_out((A.Wr + 31) / 32, (A.Hr + 7) / 8, B), g_cen((A.Ws + 31) / 32, (A.Hs + 7) / 8, B);
    dim3 g_px((W + 31) / 32, (H + 7) / 8, B);
    int dev = 0, nsm = 148;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    const size_t nrec4 = C * kRecG2;
    centre_records_kernel<<<(unsigned)((nrec4 + 255) / 256), 256, 0, st>>>(A);
    if (pixel_x2) {
        if ((e = cudaFuncSetAttribute(recon_grad_pixel_x2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(2 * rg_smem))) != cudaSuccess)
            return e;
        const int ntiles = (int)(g_out.x * g_out.y * g_out.z);
        recon_grad_pixel_x2_kernel<<<min(ntiles, 2 * nsm), 256, 2 * rg_smem, st>>>(A, g_out.x, g_out.y, ntiles,
                                                                                 (int)(rg_smem / sizeof(float4)));
    } else {
        recon_grad_pixel_kernel<<<g_out, blk, 0, st>>>(A);
    }
    if (recon_centre_rows_ok(A.hw, A.sp, A.rs)) {
        const size_t rc_smem = recon_centre_smem(A.hw, A.sp, A.rs);
        if ((e = cudaFuncSetAttribute(recon_grad_centre_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)rc_smem)) != cudaSuccess)
            return e;
        recon_grad_centre_rows_kernel<<<dim3((A.Ws + kRowCentres - 1) / kRowCentres, A.Hs, B), 64, rc_smem, st>>>(
            A);
    } else {
        recon_grad_centre_kernel<<<g_cen, blk, 0, st>>>(A);
    }
    const size_t gc_smem = grad_centre_smem(A.hw, A.sp);
    if ((e = cudaFuncSetAttribute(regression_grad_centre_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)gc_smem)) != cudaSuccess)
        return e;
    regression_grad_centre_kernel<<<dim3((A.Ws + kRowCentres - 1) / kRowCentres, A.Hs, B), 64, gc_smem, st>>>(A);
    if (tap_x2) {
        if ((e = cudaFuncSetAttribute(regression_grad_tap_x2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(2 * tg_smem))) != cudaSuccess)
            return e;
        const int ntiles = (int)(g_px.x * g_px.y * g_px.z);
        regression_grad_tap_x2_kernel<<<min(ntiles, 2 * nsm), 256, 2 * tg_smem, st>>>(A, g_px.x, g_px.y, ntiles,
                                                                                    (int)(tg_smem / sizeof(float4)));
    } else {
        regression_grad_tap_kernel<<<g_px, blk, 0, st>>>(A);
    }
    variance_grad_kernel<<<dim3(g_px.x, g_px.y, 2 * B), blk, 0, st>>>(A);
    assemble_grad_kernel<<<dim3(g_px.x, g_px.y, 2 * B), blk, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace cd
