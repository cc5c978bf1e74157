// Window rows of a row of regression centres, staged in shared memory.
//
// A CTA that owns kRowCentres consecutive centres of one centre row streams
// the rows of their windows through shared-memory row slots.  A slot holds,
// per pixel of the row segment the windows cover, four float4 groups
//   g0 = (imga.xyz, varA)  g1 = (imgb.xyz, varB)
//   g2 = (albedo.xyz, sdA) g3 = (normal.xyz, sdB)
// with positions de-interleaved by the sparsity (position p at
// (p % s) * q + p / s), so 32 lanes whose centres are s pixels apart read 32
// consecutive float4s.  Used by the forward regression (regression.cu) and
// the centre-side pass of its backward (regression_grad.cu).
#pragma once
#include <cuda_runtime.h>
#include "cd_common.cuh"

namespace cd {

constexpr int kRowCentres = 32;

struct RowGeom {
    int rw;      // row segment width in pixels
    int q;       // de-interleave stride
    int npos;    // positions per group (q * sparsity)
};

__host__ __device__ inline RowGeom row_geom(int hw, int sp)
{
    RowGeom g;
    g.rw = (kRowCentres - 1) * sp + 2 * hw + 1;
    g.q = (g.rw + sp - 1) / sp;
    g.npos = g.q * sp;
    return g;
}

CD_DEV void cp_async4(float *dst, const float *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
CD_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> CD_DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

CD_DEV int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

// Column of every row position (reflect-101; positions past the reflect
// range feed no valid centre and are clamped only to stay in bounds) and its
// de-interleaved slot index, for the segment starting at column x0.
CD_DEV void row_positions(int *pos_gx, int *pos_dst, const RowGeom &g, int x0, int W, int sp, int tid, int nthreads)
{
    for (int p = tid; p < g.rw; p += nthreads) {
        pos_gx[p] = clampi(mirror(x0 + p, W), 0, W - 1);
        pos_dst[p] = (p % sp) * g.q + p / sp;
    }
}

// Copy image row gy (of one batch image; the pointers are that image's) into
// the slot at base, as the four groups.
CD_DEV void stage_window_row(float *base, const RowGeom &g, const int *pos_gx, const int *pos_dst, int gy, int W,
                             const float *imga, const float *imgb, const float *albedo, const float *normal,
                             const float *vara, const float *varb, const float *sda, const float *sdb, int tid,
                             int nthreads)
{
    const size_t row = (size_t)gy * W;
    for (int p = tid; p < g.rw; p += nthreads) {
        const size_t q = row + pos_gx[p];
        float *d = base + 4 * pos_dst[p];
        const float *a = imga + 3 * q, *c = imgb + 3 * q, *l = albedo + 3 * q, *n = normal + 3 * q;
        float *d0 = d, *d1 = d + 4 * g.npos, *d2 = d + 8 * g.npos, *d3 = d + 12 * g.npos;
        cp_async4(d0, a); cp_async4(d0 + 1, a + 1); cp_async4(d0 + 2, a + 2); cp_async4(d0 + 3, vara + q);
        cp_async4(d1, c); cp_async4(d1 + 1, c + 1); cp_async4(d1 + 2, c + 2); cp_async4(d1 + 3, varb + q);
        cp_async4(d2, l); cp_async4(d2 + 1, l + 1); cp_async4(d2 + 2, l + 2); cp_async4(d2 + 3, sda + q);
        cp_async4(d3, n); cp_async4(d3 + 1, n + 1); cp_async4(d3 + 2, n + 2); cp_async4(d3 + 3, sdb + q);
    }
}

}  // namespace cd
