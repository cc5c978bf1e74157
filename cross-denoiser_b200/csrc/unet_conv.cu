// 3x3 convolutions of the kernel-predicting U-Net on the tensor cores
// (tcgen05, bf16 operands, fp32 accumulation in TMEM).
//
// Layer semantics: Keras Conv2D(kernel_size=3, padding='same') as the
// reference builds them (scripts/main.py:83-99): cross-correlation with zero
// padding, kernel layout [ky][kx][cin][cout], bias, ReLU.  The same kernel
// computes the input gradient (dgrad) of such a layer, as the convolution of
// the output gradient with the flipped, transposed kernel.
//
// Implicit GEMM.  A CTA owns R output rows x 128 pixels.  Its R + 2 input
// rows (131 pixels: x0-1 .. x0+129) are staged in shared memory as chunk
// planes: plane c of a row holds channels 8c..8c+7 of every pixel, 16 bytes
// per pixel.  For output row r the MMA is
//     D_r[128 px x NOUT] += A[128 px x 16] * B_s[NOUT x 16]^T   per K step s,
// where A is a 16-byte-shifted view of a staged row (the tap's kx shift) and
// its 16 K columns are two chunks: either chunks c, c+1 of one tap (LBO =
// plane size) or the same chunk of taps kx, kx+1 (LBO = 16 bytes: the second
// chunk is the next pixel).  The host builds the K-step table; the packed B
// operand holds the matching weights (zero where a step's half is unused).
// One thread issues all R x steps MMAs, commits them to an mbarrier, and the
// four warps read their 32 TMEM lanes (one pixel each) for the epilogue.
//
// Staging.  Activations are row-chunk planes (unet.cuh), so every staged
// (row, chunk) plane is one contiguous row segment in global memory: one
// bulk copy (cp.async.bulk, 16 bytes per pixel), with the pixels and rows
// outside the image copied from a page of zeros.  Every byte of the staged
// planes is written by exactly one copy, so the mbarrier's transaction count
// is the planes' total size.
#include <atomic>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "tc_sm100.cuh"
#include "unet.cuh"
#include "unet_ops.cuh"
#include "tma.cuh"

namespace cd {
namespace unet {
namespace {

constexpr int kPx = 128;                    // pixels per MMA (M)
constexpr int kStagePx = kPx + 3;           // staged pixels per row
constexpr int kPlane = kStagePx * 16;       // bytes per chunk plane
constexpr int kWaitIter = 1 << 22;          // bounded mbarrier polls

__host__ __device__ inline int b_bytes(int nsteps, int nout) { return nsteps * 2 * nout * 16; }

// Source of the zeros staged for pixels and rows outside the image (never
// written; at least one plane long).
constexpr int kZeroBytes = 4096;
static_assert(kZeroBytes >= kPlane, "the zero page covers a staged plane");
__device__ __align__(128) uint8_t g_zero_page[kZeroBytes] = {0};

// Stage pixels [xa, xa + n) of one row-chunk plane into dst (16 bytes per
// pixel) with bulk copies on `bar`: the pixels inside [0, W) from `row` (the
// plane's pixel 0; null for a row outside the image), the rest from the zero
// page.  Writes exactly n * 16 bytes.
__device__ __forceinline__ void stage_plane(uint8_t *dst, const __nv_bfloat16 *row, int xa, int n, int W,
                                            uint64_t *bar)
{
    int lo = xa, hi = xa;   // [lo, hi): the pixels copied from the image
    if (row) {
        lo = min(max(xa, 0), xa + n);
        hi = max(min(xa + n, W), lo);
    }
    if (lo > xa) tc::bulk_load(dst, g_zero_page, (uint32_t)(lo - xa) * 16u, bar);
    if (hi > lo) tc::bulk_load(dst + (size_t)(lo - xa) * 16, row + (size_t)lo * 8, (uint32_t)(hi - lo) * 16u, bar);
    if (xa + n > hi) tc::bulk_load(dst + (size_t)(hi - xa) * 16, g_zero_page, (uint32_t)(xa + n - hi) * 16u, bar);
}

// Dynamic shared memory to request so that no more CTAs share an SM than
// its 512 TMEM columns hold (228 KB of shared memory per SM): a CTA that
// cannot allocate would otherwise wait in tcgen05.alloc.
inline size_t smem_for_tmem(size_t need, int cols)
{
    const int per_sm = 512 / cols;
    const size_t cap = (size_t)233472 / (size_t)(per_sm + 1) + 1024;
    return need > cap ? need : cap;
}

__host__ __device__ inline size_t align128(size_t n) { return (n + 127) & ~(size_t)127; }
__host__ __device__ inline size_t align1k(size_t n) { return (n + 1023) & ~(size_t)1023; }

__host__ __device__ inline size_t conv_smem(int nsteps, int nout, int c0, int c1, int R)
{
    return (size_t)b_bytes(nsteps, nout) + align128((size_t)(R + 2) * c0 * kPlane) +
           align128((size_t)(R + 2) * c1 * kPlane) + 16;
}

// TMEM columns of a CTA: R row groups of NOUT accumulators, or, ky-stacked,
// R + 4 (input row i's MMAs write groups i .. i + 2, i = 0 .. R + 1; output
// row r is group r + 2), rounded up to a power of two >= 32.
template <int NOUT, int R, bool KYN>
__host__ __device__ constexpr int conv_cols()
{
    constexpr int n = KYN ? (R + 4) * NOUT : R * NOUT;
    return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512;
}

// Epilogue of one output row for the pixel x of this thread: bias, ReLU,
// the ReLU derivative of the layer below (dgrad), bf16 stores, and the fused
// 2x2 max pooling over rows (r - 1, r) of a tile whose first row is even
// (prev carries row r - 1; odd = x & 1, the pooled pair is this lane and
// lane ^ 1).  Every lane of the warp calls it (the pooling shuffles).
// bias: the caller's registers, or null to read P.bias here (kernels with
// wide rows keep registers for the accumulators).
template <int NOUT>
__device__ __forceinline__ void conv_out_row(const ConvParams &P, float (&v)[NOUT], const float *bias,
                                             float (&prev)[NOUT], int b, int x, int y, int r, int odd)
{
    const bool inside = x < P.W && y < P.H;
    const int yi = inside ? y : 0, xi = inside ? x : 0;
    if (bias) {
#pragma unroll
        for (int j = 0; j < NOUT; ++j) v[j] += bias[j];
    } else if (P.bias) {
#pragma unroll
        for (int j = 0; j < NOUT; ++j) v[j] += __ldg(P.bias + j);
    }
    if (P.relu) {
#pragma unroll
        for (int j = 0; j < NOUT; ++j) v[j] = fmaxf(v[j], 0.f);
    }
    if (inside) {
        // dgrad: multiply by the ReLU derivative of the layer below
        // (mask0 / mask1 laid out like dst0 / dst1; null = no ReLU)
#pragma unroll
        for (int c = 0; c < NOUT / 8; ++c) {
            if (c >= P.d0 + P.d1) break;
            const __nv_bfloat16 *m =
                c < P.d0 ? (P.mask0 ? P.mask0 + act_idx(b, yi, c, xi, P.H, P.W, P.d0) * 8 : nullptr)
                         : (P.mask1 ? P.mask1 + act_idx(b, yi, c - P.d0, xi, P.H, P.W, P.d1) * 8 : nullptr);
            if (!m) continue;
            const uint4 raw = *reinterpret_cast<const uint4 *>(m);
            const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&raw);
#pragma unroll
            for (int e = 0; e < 8; ++e)
                if (!(__bfloat162float(mb[e]) > 0.f)) v[8 * c + e] = 0.f;
        }
    }
    if (inside) {
#pragma unroll
        for (int c = 0; c < NOUT / 8; ++c) {
            if (c >= P.d0 + P.d1) break;
            uint4 o;
            __nv_bfloat162 *ob = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
            for (int e = 0; e < 4; ++e) ob[e] = __floats2bfloat162_rn(v[8 * c + 2 * e], v[8 * c + 2 * e + 1]);
            __nv_bfloat16 *d = c < P.d0 ? P.dst0 + act_idx(b, yi, c, xi, P.H, P.W, P.d0) * 8
                                        : P.dst1 + act_idx(b, yi, c - P.d0, xi, P.H, P.W, P.d1) * 8;
            *reinterpret_cast<uint4 *>(d) = o;
        }
    }
    if (P.pool) {
        // fused 2x2 max pooling (rows y0 + r - 1, y0 + r; lanes x, x ^ 1),
        // on the bf16-rounded outputs, as the stored activations are
        if (r & 1) {
#pragma unroll
            for (int j = 0; j < NOUT; ++j) {
                float m = fmaxf(__bfloat162float(__float2bfloat16_rn(prev[j])),
                                __bfloat162float(__float2bfloat16_rn(v[j])));
                m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
                prev[j] = m;
            }
            const int py = y / 2, px = x / 2, PH = P.H / 2, PW = P.W / 2;
            if (!odd && py < PH && px < PW) {
#pragma unroll
                for (int c = 0; c < NOUT / 8; ++c) {
                    if (c >= P.d0) break;
                    uint4 o;
                    __nv_bfloat162 *ob = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        ob[e] = __floats2bfloat162_rn(prev[8 * c + 2 * e], prev[8 * c + 2 * e + 1]);
                    *reinterpret_cast<uint4 *>(P.pool + act_idx(b, py, c, px, PH, PW, P.d0) * 8) = o;
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < NOUT; ++j) prev[j] = v[j];
        }
    }
}

// ky-stacked form: D[128 px x 3 NOUT] += A_i[128 x 16] * B_s[3 NOUT x 16]^T
// for staged input row i and K step s, with B_s's three NOUT-row blocks the
// taps ky = 2, 1, 0 and D the TMEM groups i, i + 1, i + 2: output row r
// (group r + 2) receives ky = 0 from input row r, ky = 1 from r + 1 and
// ky = 2 from r + 2, accumulating in place (every MMA accumulates into
// zero-initialised TMEM).  Compared with one MMA per output row and tap,
// (R + 2) / (3 R) of the MMAs, each N = 3 NOUT wide (an MMA of M = 128,
// K = 16 costs about the same for any N up to 64).
// NST > 0 (per-row form): P.nsteps as a template parameter, so that the
// MMA thread builds every step's descriptors once, in registers, and issues
// the R x NST MMAs without rebuilding them.
template <int NOUT, int R, bool KYN, int NST = 0>
__global__ void __launch_bounds__(128) conv3x3_kernel(const ConvParams P)
{
    extern __shared__ __align__(128) uint8_t smem[];
    constexpr int kCols = conv_cols<NOUT, R, KYN>();
    static_assert((KYN ? (R + 4) * NOUT : R * NOUT) <= 512, "TMEM holds 512 columns");
    constexpr int kRowsB = KYN ? 3 * NOUT : NOUT;   // B operand rows per step half
    const int tid = threadIdx.x, warp = tid >> 5;
    const int x0 = blockIdx.x * kPx, y0 = blockIdx.y * R, b = blockIdx.z;
    const int bb = b_bytes(P.nsteps, kRowsB);
    // [packed weights][source 0 rows][source 1 rows], blocks 128-byte aligned
    const size_t blk0 = align128((size_t)(R + 2) * P.c0 * kPlane), blk1 = align128((size_t)(R + 2) * P.c1 * kPlane);
    uint8_t *sB = smem;
    uint8_t *sA0 = smem + bb;
    uint8_t *sA1 = sA0 + blk0;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sA1 + blk1);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);

    // per input source, planes [row][chunk][131 px][8 ch] (zeros outside the
    // image), and the packed weights: bulk copies on one mbarrier
    if (warp == 0) tc::tmem_alloc(tslot, kCols);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_async_smem();
    }
    __syncthreads();   // barrier initialised before the copies are issued and waited on
    if (warp == 0) {
        const int lane = tid & 31, nch = P.c0 + P.c1;
        if (lane == 0) {
            const uint32_t bytes = (uint32_t)bb + (uint32_t)((R + 2) * nch * kPlane);
            tc::mbar_expect_tx(bar, bytes);
            tc::bulk_load(sB, P.wpack, (uint32_t)bb, bar);
        }
        __syncwarp();   // the transaction count is raised before any copy lands
        for (int i = lane; i < (R + 2) * nch; i += 32) {
            const int r = i / nch, c = i - r * nch, gy = y0 - 1 + r;
            const bool s1 = c >= P.c0;
            const int cs = s1 ? c - P.c0 : c, ns = s1 ? P.c1 : P.c0;
            uint8_t *dst = (s1 ? sA1 : sA0) + (size_t)(r * ns + cs) * kPlane;
            const __nv_bfloat16 *row =
                gy >= 0 && gy < P.H ? (s1 ? P.src1 : P.src0) + act_idx(b, gy, cs, 0, P.H, P.W, ns) * 8 : nullptr;
            stage_plane(dst, row, x0 - 1, kStagePx, P.W, bar);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    const bool staged = __syncthreads_and(tc::mbar_wait(bar, 0, kWaitIter)) != 0;
    tc::fence_after_sync();
    const uint32_t tbase = *tslot;
    if (!staged) {
        if (tid == 0) atomicExch(P.err, 1);
        tc::fence_before_sync();
        __syncthreads();
        if (warp == 0) tc::tmem_dealloc(tbase, kCols);
        return;
    }
    if (KYN) {
        // zero the accumulators: each warp its 32 lanes, every group
        const uint32_t lanes = tbase + ((uint32_t)(warp * 32) << 16);
        for (int col = 0; col < (R + 4) * NOUT; col += 16) tc::tmem_st16_zero(lanes + col);
        tc::tmem_wait_st();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
    }
    if (tid == 0) {
        const uint32_t a0 = tc::smem_u32(sA0), a1 = tc::smem_u32(sA1), b0 = tc::smem_u32(sB);
        if (KYN) {
            const uint32_t idesc = tc::idesc_bf16(kPx, 3 * NOUT);
            for (int i = 0; i < R + 2; ++i)
                for (int s = 0; s < P.nsteps; ++s) {
                    const KStep st = P.steps[s];
                    const uint32_t base = st.src ? a1 + (uint32_t)(i * P.c1) * kPlane : a0 + (uint32_t)(i * P.c0) * kPlane;
                    const uint64_t ad = tc::sdesc(base + st.a_off, st.a_lbo, 128);
                    const uint64_t bd = tc::sdesc(b0 + (uint32_t)(s * 2 * kRowsB * 16), kRowsB * 16, 128);
                    tc::mma_bf16(tbase + i * NOUT, ad, bd, idesc, 1u);
                }
        } else if (NST > 0) {
            constexpr int kN = NST > 0 ? NST : 1;
            const uint32_t idesc = tc::idesc_bf16(kPx, NOUT);
            // row-0 A descriptor of each step, its row stride (16-byte units), B descriptor
            uint64_t ad[kN], bd[kN];
            uint32_t rs[kN];
#pragma unroll
            for (int s = 0; s < kN; ++s) {
                const KStep st = P.steps[s];
                const uint32_t base = st.src ? a1 + (uint32_t)(st.ky * P.c1) * kPlane : a0 + (uint32_t)(st.ky * P.c0) * kPlane;
                ad[s] = tc::sdesc(base + st.a_off, st.a_lbo, 128);
                rs[s] = (uint32_t)((st.src ? P.c1 : P.c0) * kPlane) >> 4;
                bd[s] = tc::sdesc(b0 + (uint32_t)(s * 2 * NOUT * 16), NOUT * 16, 128);
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int s = 0; s < kN; ++s)
                    tc::mma_bf16(tbase + r * NOUT, ad[s] + (uint64_t)(r * rs[s]), bd[s], idesc, s > 0 ? 1u : 0u);
        } else {
            const uint32_t idesc = tc::idesc_bf16(kPx, NOUT);
            for (int r = 0; r < R; ++r)
                for (int s = 0; s < P.nsteps; ++s) {
                    const KStep st = P.steps[s];
                    const uint32_t base = st.src ? a1 + (uint32_t)((r + st.ky) * P.c1) * kPlane
                                                 : a0 + (uint32_t)((r + st.ky) * P.c0) * kPlane;
                    const uint64_t ad = tc::sdesc(base + st.a_off, st.a_lbo, 128);
                    const uint64_t bd = tc::sdesc(b0 + (uint32_t)(s * 2 * NOUT * 16), NOUT * 16, 128);
                    tc::mma_bf16(tbase + r * NOUT, ad, bd, idesc, s > 0 ? 1u : 0u);
                }
        }
        tc::commit(bar);
    }
    // the commit completes the barrier's second phase (parity 1)
    const bool done = __syncthreads_and(tc::mbar_wait(bar, 1, kWaitIter)) != 0;   // uniform across the CTA
    tc::fence_after_sync();
    if (!done) {
        if (tid == 0) atomicExch(P.err, 2);
    } else {
        const int x = x0 + tid;
        const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
        float prev[NOUT];
        for (int r = 0; r < R; ++r) {
            float v[NOUT];
#pragma unroll
            for (int j = 0; j < NOUT; j += 16) tc::tmem_ld16(lane_base + (KYN ? r + 2 : r) * NOUT + j, v + j);
            conv_out_row<NOUT>(P, v, nullptr, prev, b, x, y0 + r, r, tid & 1);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, kCols);
}

template <int NOUT, int R, bool KYN, int NST = 0>
cudaError_t launch_t(const ConvParams &P, int B, cudaStream_t st)
{
    constexpr int kCols = conv_cols<NOUT, R, KYN>();
    const size_t smem = smem_for_tmem(conv_smem(P.nsteps, KYN ? 3 * NOUT : NOUT, P.c0, P.c1, R), kCols);
    cudaError_t e = cudaFuncSetAttribute(conv3x3_kernel<NOUT, R, KYN, NST>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((P.W + kPx - 1) / kPx, (P.H + R - 1) / R, B);
    conv3x3_kernel<NOUT, R, KYN, NST><<<grid, 128, smem, st>>>(P);
    return cudaGetLastError();
}

// Per-row form with the step count as a template parameter for the
// network's 32- and 48-output layers (5, 6, 9 or 18 steps), the run-time
// loop otherwise.
template <int NOUT, int R>
cudaError_t launch_rows(const ConvParams &P, int B, cudaStream_t st)
{
    switch (P.nsteps) {
    case 5: return launch_t<NOUT, R, false, 5>(P, B, st);
    case 6: return launch_t<NOUT, R, false, 6>(P, B, st);
    case 9: return launch_t<NOUT, R, false, 9>(P, B, st);
    case 18: return launch_t<NOUT, R, false, 18>(P, B, st);
    default: return launch_t<NOUT, R, false>(P, B, st);
    }
}

// Persistent, pipelined form of the ky-stacked convolution.  The same MMAs
// per tile (R output rows x 128 pixels) as conv3x3_kernel<NOUT, R, true>,
// with the roles split over warps so that staging, tensor-core work and the
// epilogue of different tiles overlap: warp 0 stages tile i into ring slot
// i % S (bulk copies; the packed weights once per CTA), lane 0 of warp 1
// issues the tile's MMAs into TMEM accumulator buffer i % 2 and commits them
// to the slot's "empty" and the buffer's "full" barriers, and warps 2..5
// (TMEM lanes = pixels) run the epilogue of the buffer, zero it and hand it
// back through its "empty" barrier.  The epilogue is the longest of the
// three per tile, so it has two warps per TMEM lane quadrant, one per pair
// of output rows (the fused pooling pairs rows 2k, 2k + 1), and two CTAs
// share an SM where their rings fit half of its shared memory.  Every wait
// is bounded.
constexpr int kPipeEpiWarps = 8;
constexpr int kPipeThreads = 64 + 32 * kPipeEpiWarps;
constexpr int kPipeSmem = 225 * 1024;     // one CTA per SM
constexpr int kPipeSmem2 = 112 * 1024;    // two CTAs per SM
constexpr int kPipeMaxSlots = 8;

struct ConvPipePlan {
    uint32_t wbytes;   // packed weights (B operand), rounded up to 1 KB
    uint32_t blk0;     // source 0 rows of a slot
    uint32_t stage;    // bytes per ring slot
    uint32_t tx;       // bytes the copies of one slot deliver
    int S;             // ring slots
    size_t smem;
};

inline ConvPipePlan conv_pipe_plan(int nsteps, int nout_rows, int c0, int c1, int R, int smem_cap)
{
    ConvPipePlan p{};
    p.wbytes = (uint32_t)align1k((size_t)b_bytes(nsteps, nout_rows));
    p.blk0 = (uint32_t)align128((size_t)(R + 2) * c0 * kPlane);
    p.stage = (uint32_t)align1k(p.blk0 + align128((size_t)(R + 2) * c1 * kPlane));
    p.tx = (uint32_t)((R + 2) * (c0 + c1) * kPlane);
    const long room = (long)smem_cap - (long)p.wbytes - 1024;
    const int S = room > 0 ? (int)(room / (long)p.stage) : 0;
    p.S = S > kPipeMaxSlots ? kPipeMaxSlots : S;
    p.smem = (size_t)p.wbytes + (size_t)p.S * p.stage + 1024;
    return p;
}

// NST: K steps per input row (P.nsteps), a template parameter so that the
// MMA thread keeps every step's descriptors in registers: one thread issues
// all MMAs, and with descriptors rebuilt per MMA its instruction chain, not
// the tensor core, set the pace.
template <int NOUT, int R, int NST>
__global__ void __launch_bounds__(kPipeThreads, 2)
    conv3x3_pipe_kernel(const ConvParams P, const ConvPipePlan pl, int ntx, int nty, int ntiles)
{
    extern __shared__ __align__(128) uint8_t smem[];
    constexpr int kRowsB = 3 * NOUT;
    constexpr int kGrp = (R + 4) * NOUT;   // TMEM columns of one accumulator buffer
    constexpr int kCols = 2 * kGrp <= 32 ? 32 : 2 * kGrp <= 64 ? 64 : 2 * kGrp <= 128 ? 128 : 2 * kGrp <= 256 ? 256 : 512;
    static_assert(2 * kGrp <= 256, "two CTAs' accumulator buffers fit TMEM");
    static_assert(R == 2 * (kPipeEpiWarps / 4), "one epilogue warp per lane quadrant and row pair");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int S = pl.S;
    uint8_t *sB = smem;
    uint8_t *ring = smem + pl.wbytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + (size_t)S * pl.stage);
    uint64_t *empty = full + S;
    uint64_t *tfull = empty + S;    // [2] accumulator buffer written
    uint64_t *tempty = tfull + 2;   // [2] accumulator buffer read and zeroed
    uint64_t *wbar = tempty + 2;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(wbar + 1);

    if (warp == 1) tc::tmem_alloc(tslot, kCols);
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int k = 0; k < 2; ++k) {
            tc::mbar_init(&tfull[k], 1);
            tc::mbar_init(&tempty[k], kPipeEpiWarps);
        }
        tc::mbar_init(wbar, 1);
        tc::fence_async_smem();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *tslot;
    // both accumulator buffers start at zero (every MMA accumulates)
    if (warp >= 2) {
        const uint32_t lanes = tbase + ((uint32_t)((warp & 3) * 32) << 16);
        const int rp = (warp - 2) >> 2;
        for (int k = 0; k < 2; ++k)
            for (int col = rp * (kGrp / 2); col < (rp + 1) * (kGrp / 2); col += 16)
                tc::tmem_st16_zero(lanes + (uint32_t)(k * kGrp + col));
        tc::tmem_wait_st();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();

    const int first = blockIdx.x, stride = gridDim.x;
    int ntile = 0;
    for (int t = first; t < ntiles; t += stride) ++ntile;
    bool ok = true;

    if (warp == 0) {
        // ---- producer: one bulk copy per chunk plane row (zeros outside
        // the image), the packed weights once ----
        const uint32_t bb = (uint32_t)b_bytes(P.nsteps, kRowsB);
        if (lane == 0) {
            tc::mbar_expect_tx(wbar, bb);
            tc::bulk_load(sB, P.wpack, bb, wbar);
        }
        const int nch = P.c0 + P.c1;
        int i = 0;
        for (; i < ntile; ++i) {
            const int s = i % S, tile = first + i * stride;
            if (i >= S) {
                bool got = true;
                if (lane == 0) got = tc::mbar_wait(&empty[s], (uint32_t)(i / S - 1) & 1u, kWaitIter);
                if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) {
                    ok = false;
                    break;
                }
            }
            const int tx = tile % ntx, ty = (tile / ntx) % nty, b = tile / (ntx * nty);
            const int x0 = tx * kPx, y0 = ty * R;
            uint8_t *sA0 = ring + (size_t)s * pl.stage, *sA1 = sA0 + pl.blk0;
            if (lane == 0) tc::mbar_expect_tx(&full[s], pl.tx);
            __syncwarp();   // the transaction count is raised before any copy lands
            for (int q = lane; q < (R + 2) * nch; q += 32) {
                const int r = q / nch, c = q - r * nch, gy = y0 - 1 + r;
                const bool s1 = c >= P.c0;
                const int cs = s1 ? c - P.c0 : c, ns = s1 ? P.c1 : P.c0;
                uint8_t *dst = (s1 ? sA1 : sA0) + (size_t)(r * ns + cs) * kPlane;
                const __nv_bfloat16 *row =
                    gy >= 0 && gy < P.H ? (s1 ? P.src1 : P.src0) + act_idx(b, gy, cs, 0, P.H, P.W, ns) * 8 : nullptr;
                stage_plane(dst, row, x0 - 1, kStagePx, P.W, &full[s]);
            }
        }
        // every copy issued has landed before the CTA may exit
        if (lane == 0) {
            tc::mbar_wait(wbar, 0, kWaitIter);
            for (int s = 0; s < S && s < i; ++s)
                tc::mbar_wait(&full[s], (uint32_t)((i - s + S - 1) / S - 1) & 1u, kWaitIter);
        }
    } else if (warp == 1) {
        // ---- MMA issue (one thread) ----
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16(kPx, kRowsB);
            // per K step: A descriptor of row 0 relative to a slot (start
            // field = byte offset / 16), its row stride in 16-byte units,
            // and the B descriptor
            uint64_t ad[NST], bd[NST];
            uint32_t rs[NST];
            const uint32_t b0 = tc::smem_u32(sB);
#pragma unroll
            for (int k = 0; k < NST; ++k) {
                const KStep st = P.steps[k];
                ad[k] = tc::sdesc((st.src ? pl.blk0 : 0u) + (uint32_t)st.a_off, st.a_lbo, 128);
                rs[k] = (uint32_t)((st.src ? P.c1 : P.c0) * kPlane) >> 4;
                bd[k] = tc::sdesc(b0 + (uint32_t)(k * 2 * kRowsB * 16), kRowsB * 16, 128);
            }
            ok = tc::mbar_wait(wbar, 0, kWaitIter);
            for (int i = 0; ok && i < ntile; ++i) {
                const int s = i % S, buf = i & 1;
                if (!tc::mbar_wait(&full[s], (uint32_t)(i / S) & 1u, kWaitIter) ||
                    (i >= 2 && !tc::mbar_wait(&tempty[buf], (uint32_t)(i / 2 - 1) & 1u, kWaitIter))) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                // slot base added to the start field (addresses stay below 2^18)
                const uint64_t sbase = (uint64_t)(tc::smem_u32(ring + (size_t)s * pl.stage) >> 4);
                const uint32_t acc = tbase + (uint32_t)(buf * kGrp);
                // rows, then K steps: the per-tile kernel's accumulation order
                uint64_t at[NST];
#pragma unroll
                for (int k = 0; k < NST; ++k) at[k] = ad[k] + sbase;
#pragma unroll
                for (int r = 0; r < R + 2; ++r)
#pragma unroll
                    for (int k = 0; k < NST; ++k)
                        tc::mma_bf16(acc + r * NOUT, at[k] + (uint64_t)(r * rs[k]), bd[k], idesc, 1u);
                tc::commit(&empty[s]);
                tc::commit(&tfull[buf]);
            }
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    } else {
        // ---- epilogue: TMEM lane m = pixel x0 + m, output rows 2 rp, 2 rp + 1 ----
        const int m = (warp & 3) * 32 + lane, rp = (warp - 2) >> 2;
        const uint32_t lanes = tbase + ((uint32_t)((warp & 3) * 32) << 16);
        float bias[NOUT];
#pragma unroll
        for (int j = 0; j < NOUT; ++j) bias[j] = P.bias ? __ldg(P.bias + j) : 0.f;   // zeros: no bias
        for (int i = 0; i < ntile; ++i) {
            const int buf = i & 1, tile = first + i * stride;
            bool got = true;
            if (lane == 0) got = tc::mbar_wait(&tfull[buf], (uint32_t)(i / 2) & 1u, kWaitIter);
            if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) {
                ok = false;
                break;
            }
            tc::fence_after_sync();
            const int tx = tile % ntx, ty = (tile / ntx) % nty, b = tile / (ntx * nty);
            const int x = tx * kPx + m, y0 = ty * R;
            const uint32_t accl = lanes + (uint32_t)(buf * kGrp);
            float prev[NOUT];
#pragma unroll
            for (int r = 2 * rp; r < 2 * rp + 2; ++r) {
                float v[NOUT];
#pragma unroll
                for (int j = 0; j < NOUT; j += 16) tc::tmem_ld16(accl + (r + 2) * NOUT + j, v + j);
                conv_out_row<NOUT>(P, v, bias, prev, b, x, y0 + r, r, lane & 1);
            }
            // zero this warp's share of the buffer: its lanes, a column
            // range per row pair
            for (int col = rp * (kGrp / 2); col < (rp + 1) * (kGrp / 2); col += 16) tc::tmem_st16_zero(accl + col);
            tc::tmem_wait_st();
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(&tempty[buf])) : "memory");
        }
    }
    ok = __syncthreads_and(ok) != 0;
    if (!ok && tid == 0) atomicExch(P.err, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) tc::tmem_dealloc(tbase, kCols);
}

// per_sm: CTAs per SM the plan's shared memory allows (1 or 2)
template <int NOUT, int R, int NST>
cudaError_t launch_pipe_t(const ConvParams &P, const ConvPipePlan &pl, int per_sm, int B, cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(conv3x3_pipe_kernel<NOUT, R, NST>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem);
    if (e != cudaSuccess) return e;
    const int ntx = (P.W + kPx - 1) / kPx, nty = (P.H + R - 1) / R, ntiles = B * ntx * nty;
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = ntiles < per_sm * nsm ? ntiles : per_sm * nsm;
    conv3x3_pipe_kernel<NOUT, R, NST><<<grid, kPipeThreads, pl.smem, st>>>(P, pl, ntx, nty, ntiles);
    return cudaGetLastError();
}

// The step counts of the network's 16-output layers: 2 (one chunk), 3 (a
// chunk pair), 5, 6, 9; others return cudaErrorNotSupported.
template <int NOUT, int R>
cudaError_t launch_pipe(const ConvParams &P, const ConvPipePlan &pl, int per_sm, int B, cudaStream_t st)
{
    switch (P.nsteps) {
    case 2: return launch_pipe_t<NOUT, R, 2>(P, pl, per_sm, B, st);
    case 3: return launch_pipe_t<NOUT, R, 3>(P, pl, per_sm, B, st);
    case 5: return launch_pipe_t<NOUT, R, 5>(P, pl, per_sm, B, st);
    case 6: return launch_pipe_t<NOUT, R, 6>(P, pl, per_sm, B, st);
    case 9: return launch_pipe_t<NOUT, R, 9>(P, pl, per_sm, B, st);
    default: return cudaErrorNotSupported;
    }
}
bool pipe_steps_supported(int n) { return n == 2 || n == 3 || n == 5 || n == 6 || n == 9; }

// Packed B operand: per step s, half h, conv output row n, element e
// (dst[((s * 2 + h) * nout + n) * 8 + e]) the weight of tap (ky, kx) from
// conv input channel 8 * chunk + e to conv output channel n; in a ky-stacked
// table the rows are 3 * nout, row n' holding tap ky = 2 - n' / nout of
// output channel n' % nout.
__device__ __forceinline__ void pack_one(const float *__restrict__ w, __nv_bfloat16 *__restrict__ dst,
                                         const PackTable &T, int i)
{
    const int rows = T.stacked ? 3 * T.nout : T.nout;
    if (i >= T.nsteps * 2 * rows * 8) return;
    const int e = i & 7, nr = (i >> 3) % rows, h = (i / (8 * rows)) & 1, s = i / (16 * rows);
    StepHalf hf = T.half[s][h];
    int n = nr;
    if (T.stacked) {
        hf.ky = 2 - nr / T.nout;   // rows [0, n): ky 2, [n, 2n): ky 1, [2n, 3n): ky 0
        n = nr % T.nout;
    }
    float v = 0.f;
    if (hf.chunk >= 0) {
        const int ci = 8 * hf.chunk + e;
        if (!T.dgrad) {
            if (ci < T.cin && n < T.cout) v = w[((hf.ky * 3 + hf.kx) * T.cin + ci) * T.cout + n];
        } else {
            // conv of dZ: input channel = layer output ci, output channel = layer input n, flipped taps
            if (ci < T.cout && n < T.cin) v = w[(((2 - hf.ky) * 3 + (2 - hf.kx)) * T.cin + n) * T.cout + ci];
        }
    }
    dst[i] = __float2bfloat16_rn(v);
}

__global__ void pack_kernel(const float *__restrict__ w, __nv_bfloat16 *__restrict__ dst, const PackTable T)
{
    pack_one(w, dst, T, blockIdx.x * blockDim.x + threadIdx.x);
}

// grid row j packs job j
__global__ void pack_jobs_kernel(const __grid_constant__ PackJobs J)
{
    const PackJob &j = J.job[blockIdx.y];
    pack_one(j.w, j.dst, j.T, blockIdx.x * blockDim.x + threadIdx.x);
}

// Weight gradient.  D_tap[cin x cout] = sum_p X[p + tap][cin] dZ[p][cout]:
// M = input channels (128 rows: the chunk planes of X from chunk 0 on), N =
// output channels padded to NZ, K = 16 consecutive pixels per MMA; both
// operands MN-major (channels contiguous, pixels 16 bytes apart).  Nine
// accumulators, one per tap.  Each staged row carries, after its nch chunk
// planes, a plane of ones, so row 8 * nch of the centre tap's accumulator is
// sum_p dZ[p][cout], the bias gradient; rows past it read other staged data
// and are discarded.  A CTA covers R rows x 128 pixels and writes its
// partial sums [9 * cin * cout weights, cout biases].
constexpr int kZPlane = kPx * 16;

__host__ __device__ inline size_t wgrad_smem(int nch, int zc, int R)
{
    return (size_t)((R + 2) * (nch + 1) + 16) * kPlane + (size_t)(R * zc + 4) * kZPlane + 16;
}

template <int NZ, int R>
__global__ void __launch_bounds__(128) wgrad_kernel(const WgradParams P)
{
    extern __shared__ __align__(128) uint8_t smem[];
    constexpr int kCols = 9 * NZ <= 256 ? 256 : 512;
    static_assert(9 * NZ <= 512, "nine accumulators of NZ columns");
    const int tid = threadIdx.x, warp = tid >> 5;
    const int x0 = blockIdx.x * kPx, y0 = blockIdx.y * R, b = blockIdx.z;
    const int tile = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    const int nch = P.xc0 + P.xc1, rs = nch + 1;   // planes per staged row (with the ones plane)
    uint8_t *sX = smem;
    uint8_t *sZ = sX + (size_t)((R + 2) * rs + 16) * kPlane;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sZ + (size_t)(R * P.zc + 4) * kZPlane);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    for (int i = tid; i < (R + 2) * nch * kStagePx; i += 128) {
        const int px = i % kStagePx, t = i / kStagePx;
        const int c = t % nch, r = t / nch;
        const int gy = y0 - 1 + r, gx = x0 - 1 + px;
        const bool in = gy >= 0 && gy < P.H && gx >= 0 && gx < P.W;
        const int yi = in ? gy : 0, xi = in ? gx : 0;
        const __nv_bfloat16 *src = c < P.xc0 ? P.x0 + act_idx(b, yi, c, xi, P.H, P.W, P.xc0) * 8
                                             : P.x1 + act_idx(b, yi, c - P.xc0, xi, P.H, P.W, P.xc1) * 8;
        tc::cp16(sX + (size_t)(r * rs + c) * kPlane + 16 * px, src, in ? 16u : 0u);
    }
    const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);   // bf16 1.0 x 8
    for (int i = tid; i < (R + 2) * kStagePx; i += 128) {
        const int px = i % kStagePx, r = i / kStagePx;
        *reinterpret_cast<uint4 *>(sX + (size_t)(r * rs + nch) * kPlane + 16 * px) = ones;
    }
    for (int i = tid; i < R * P.zc * kPx; i += 128) {
        const int px = i % kPx, t = i / kPx;
        const int c = t % P.zc, r = t / P.zc;
        const int gy = y0 + r, gx = x0 + px;
        const bool in = gy < P.H && gx < P.W;
        const __nv_bfloat16 *src = P.dz + act_idx(b, in ? gy : 0, c, in ? gx : 0, P.H, P.W, P.zc) * 8;
        tc::cp16(sZ + (size_t)(r * P.zc + c) * kZPlane + 16 * px, src, in ? 16u : 0u);
    }
    if (warp == 0) tc::tmem_alloc(tslot, kCols);
    if (tid == 0) tc::mbar_init(bar, 1);
    tc::cp_wait_all();
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *tslot;

    if (tid == 0) {
        const uint32_t idesc = tc::idesc_bf16(kPx, NZ) | (1u << 15) | (1u << 16);   // A and B MN-major
        const uint32_t ax = tc::smem_u32(sX), az = tc::smem_u32(sZ);
        for (int r = 0; r < R; ++r)
            for (int g = 0; g < kPx / 16; ++g) {
                const uint64_t bd = tc::sdesc(az + (uint32_t)(r * P.zc) * kZPlane + 256u * g, 128, kZPlane);
                for (int tap = 0; tap < 9; ++tap) {
                    const int ky = tap / 3, kx = tap - 3 * ky;
                    const uint32_t a = ax + (uint32_t)((r + ky) * rs) * kPlane + (uint32_t)(kx + 16 * g) * 16;
                    tc::mma_bf16(tbase + tap * NZ, tc::sdesc(a, 128, kPlane), bd, idesc, (r | g) ? 1u : 0u);
                }
            }
        tc::commit(bar);
    }
    const bool done = __syncthreads_and(tc::mbar_wait(bar, 0, kWaitIter)) != 0;   // uniform across the CTA
    tc::fence_after_sync();
    float *out = P.partial + (size_t)tile * (9 * P.cin * P.cout + P.cout);
    if (!done) {
        if (tid == 0) atomicExch(P.err, 1);
    } else if (warp * 32 <= 8 * nch) {
        const int m = warp * 32 + (tid & 31);
        for (int tap = 0; tap < 9; ++tap)
#pragma unroll
            for (int j = 0; j < NZ; j += 16) {
                float v[16];
                tc::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + tap * NZ + j, v);
                if (m < P.cin) {
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        if (j + q < P.cout) out[(tap * P.cin + m) * P.cout + j + q] = v[q];
                } else if (m == 8 * nch && tap == 4) {
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        if (j + q < P.cout) out[9 * P.cin * P.cout + j + q] = v[q];
                }
            }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, kCols);
}

constexpr int kWgradThreads = 192;     // persistent weight gradient: producer, MMA, 4 bias warps
constexpr int kWgradBiasWarps = 4;

constexpr int kWgradRows = 4;

template <int NZ>
cudaError_t launch_wgrad_t(const WgradParams &P, int B, cudaStream_t st)
{
    const size_t smem = smem_for_tmem(wgrad_smem(P.xc0 + P.xc1, P.zc, kWgradRows), 9 * NZ <= 256 ? 256 : 512);
    cudaError_t e = cudaFuncSetAttribute(wgrad_kernel<NZ, kWgradRows>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((P.W + kPx - 1) / kPx, (P.H + kWgradRows - 1) / kWgradRows, B);
    wgrad_kernel<NZ, kWgradRows><<<grid, 128, smem, st>>>(P);
    return cudaGetLastError();
}

// Persistent weight gradient of a 3x3 layer, two forms.
//
// Nine-tap form (T9): one MMA per input row and 16 pixels covers
// every tap,
//   D[cin x (ky, kx, cout)] += X_i^T[cin x 16 px from x0 + 16g] dZ'_i[16 px x (ky, kx, cout)]
// A is input row i (128 pixels from x0, one plane per chunk: source 0, then
// source 1), so its M groups are the chunk planes.  B is the output
// gradient staged three times per row, shifted by the horizontal tap: copy
// kx of row j holds pixels x0 + 1 - kx .. x0 + 128 - kx of output-gradient
// row y0 - 1 + j.  Planes are ordered (row, kx, chunk), so for input row i
// the rows i, i + 1, i + 2 (ky = 2, 1, 0) with their three copies are 9 zc
// consecutive planes: N = 72 zc (rounded up to 16) in one MMA.  A tcgen05
// MMA of M = 128, K = 16 costs about the same for any N up to 64 and grows
// slowly above, so this form issues a third of the MMAs of the three-tap
// form for 3 zc of the output gradient's planes per row instead of zc.
//
// Three-tap form (wider output gradients): three MMAs
// per input row and 16 pixels, one per horizontal tap kx,
//   D_kx[cin x (ky, cout)] += X_i^T[cin x 16 px from x0 + 16g + kx - 1] dZ_i[16 px x (ky, cout)]
// with input row i staged once (130 pixels from x0 - 1) and the tap a
// 16-byte (one pixel) shift of A's K start; B holds the output-gradient
// rows i - 1, i, i + 1 (ky = 2, 1, 0) as consecutive planes.
//
// In both, M = 128 rows cover the 8 x chunks input channels; rows and
// columns past the layer's channels read other staged data (or the
// shared-memory tail that the plan reserves past the last stage) and are
// discarded.  Both operands MN-major (channels contiguous, pixels 16 bytes
// apart).
//
// A tile is R input rows x 128 pixels: the output gradient's R + 2 rows from
// y0 - 1 and the input rows, one bulk copy per plane with zeros outside the
// image (stage_plane), land in a ring of S stages.  The warps specialise:
// warp 0 stages tile i into slot i % S once the slot's "empty" barrier says
// its previous MMAs and bias reads are done (all 32 lanes issue copies);
// lane 0 of warp 1 issues the tile's MMAs when the slot is full and commits
// them to "empty"; warps 2..5 sum the bias gradient (the output gradient
// over the tile's R centre rows) from the staged planes and arrive on
// "empty".  CTAs are persistent and keep their accumulators in TMEM over all
// their tiles; one partial sum per CTA, read out of TMEM by warps 2..5 at
// the end.  Every wait is bounded.
constexpr int kWgrad3Smem = 225 * 1024;
constexpr int kXPx = kPx + 2;                 // staged input pixels per row (three-tap form)
constexpr int kXPlane = kXPx * 16;
constexpr int kWgrad3Fixed = 2048;            // barriers, then the bias reduction

// MMA width (columns per MMA) and MMAs per input row and 16 pixels.
__host__ __device__ constexpr int wgrad3_n(int zc, bool t9) { return ((t9 ? 72 : 24) * zc + 15) & ~15; }
__host__ __device__ constexpr int wgrad3_mmas(bool t9) { return t9 ? 1 : 3; }

struct Wgrad3Plan {
    int R, S;         // input rows per tile, ring slots
    size_t xoff, zoff, xbytes, zbytes, stage;
    size_t extra;     // bytes past the last stage that the MMAs' operands reach
    size_t smem;
};

__host__ __device__ inline Wgrad3Plan wgrad3_stage(int xc, int zc, int R, bool t9)
{
    Wgrad3Plan p{};
    p.R = R;
    size_t a_end, b_end;   // end of the operand bytes the last row's MMAs read
    if (t9) {
        p.xbytes = (size_t)R * xc * kZPlane;
        p.zbytes = (size_t)(R + 2) * 3 * zc * kZPlane;
        p.xoff = 0;
        p.zoff = align1k(p.xbytes);
        p.stage = p.zoff + align1k(p.zbytes);
        a_end = p.xoff + (size_t)((R - 1) * xc + 16) * kZPlane;
        b_end = p.zoff + (size_t)((R - 1) * 3 * zc + wgrad3_n(zc, true) / 8) * kZPlane;
    } else {
        p.zbytes = (size_t)(R + 2) * zc * kZPlane;
        p.xbytes = (size_t)R * xc * kXPlane;
        p.zoff = 0;
        p.xoff = align1k(p.zbytes);
        p.stage = p.xoff + align1k(p.xbytes);
        a_end = p.xoff + (size_t)((R - 1) * xc + 16) * kXPlane;
        b_end = p.zoff + (size_t)((R - 1) * zc + wgrad3_n(zc, false) / 8) * kZPlane + 2 * 16;
    }
    const size_t end = a_end > b_end ? a_end : b_end;
    p.extra = end > p.stage ? align1k(end - p.stage) : 0;
    return p;
}

// Largest R (8, 4, 2, 1) that leaves at least `min_slots` ring slots (the
// nine-tap form: 3; 2-row tiles in a deeper ring measured slower, 89
// against 60 us at 1920x1080, 24 -> 8 channels).
inline Wgrad3Plan wgrad3_plan(int xc, int zc, bool t9)
{
    const int min_slots = t9 ? 3 : 4, max_slots = 6;
    Wgrad3Plan p{};
    for (int R = 8; R >= 1; R >>= 1) {
        p = wgrad3_stage(xc, zc, R, t9);
        const long room = (long)kWgrad3Smem - (long)p.extra - kWgrad3Fixed;
        const int S = room > 0 ? (int)(room / (long)p.stage) : 0;
        p.S = S > max_slots ? max_slots : S;
        p.smem = (size_t)p.S * p.stage + p.extra + kWgrad3Fixed;
        if (p.S >= min_slots) break;
    }
    return p;
}

__host__ __device__ inline int pow2_cols(int n)
{
    int c = 32;
    while (c < n) c <<= 1;
    return c;
}

template <int ZC, bool T9>
__global__ void __launch_bounds__(kWgradThreads, 1) wgrad3_kernel(const WgradParams P, const Wgrad3Plan pl, int ntx,
                                                                 int nty, int ntiles)
{
    extern __shared__ __align__(128) uint8_t smem[];
    constexpr int N = wgrad3_n(ZC, T9);
    constexpr int NMMA = wgrad3_mmas(T9);
    constexpr int kZRow = T9 ? 3 * ZC : ZC;   // output-gradient planes per staged row
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int xc0 = P.xc0, xc1 = P.xc1, xc = xc0 + xc1;
    const int R = pl.R, S = pl.S;
    const uint32_t cols = (uint32_t)pow2_cols(NMMA * N);
    const size_t stage_bytes = pl.stage;
    uint8_t *tail = smem + (size_t)S * stage_bytes + pl.extra;
    uint64_t *full = reinterpret_cast<uint64_t *>(tail);
    uint64_t *empty = full + S;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(empty + S);
    float *red = reinterpret_cast<float *>(tail + 1024);   // [4][8 * ZC]

    if (warp == 1) tc::tmem_alloc(tslot, cols);
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1 + kWgradBiasWarps);   // the MMA commit + the bias warps
        }
        tc::fence_async_smem();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *tslot;
    const int first = blockIdx.x, stride = gridDim.x;
    bool ok = true;
    int ntile = 0;   // tiles this CTA walks
    for (int t = first; t < ntiles; t += stride) ++ntile;

    float bsum[8 * ZC];
#pragma unroll
    for (int j = 0; j < 8 * ZC; ++j) bsum[j] = 0.f;

    if (warp == 0) {
        // ---- producer: all lanes issue the planes of a stage ----
        const int nz = (R + 2) * kZRow, nplanes = nz + R * xc;
        const uint32_t tx_bytes = (uint32_t)(pl.zbytes + pl.xbytes);
        int i = 0;
        for (; i < ntile; ++i) {
            const int s = i % S, tile = first + i * stride;
            if (i >= S) {
                bool got = true;
                if (lane == 0) got = tc::mbar_wait(&empty[s], (uint32_t)(i / S - 1) & 1u, kWaitIter);
                if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) {
                    ok = false;
                    break;
                }
            }
            const int tx = tile % ntx, ty = (tile / ntx) % nty, b = tile / (ntx * nty);
            const int x0 = tx * kPx, y0 = ty * R;
            uint8_t *st = smem + (size_t)s * stage_bytes;
            if (lane == 0) tc::mbar_expect_tx(&full[s], tx_bytes);
            __syncwarp();   // the transaction count is raised before any copy lands
            for (int q = lane; q < nplanes; q += 32) {
                if (q < nz) {
                    // output gradient: staged row j = image row y0 - 1 + j;
                    // nine-tap form: copy kx from pixel x0 + 1 - kx
                    const int j = q / kZRow, u = q - j * kZRow, kx = T9 ? u / ZC : 0, c = u - kx * ZC;
                    const int gy = y0 - 1 + j;
                    const __nv_bfloat16 *row =
                        gy >= 0 && gy < P.H ? P.dz + act_idx(b, gy, c, 0, P.H, P.W, ZC) * 8 : nullptr;
                    stage_plane(st + pl.zoff + (size_t)q * kZPlane, row, T9 ? x0 + 1 - kx : x0, kPx, P.W, &full[s]);
                } else {
                    // input row r, chunk c (source 0, then source 1)
                    const int u = q - nz, r = u / xc, c = u - r * xc, gy = y0 + r;
                    const bool s1 = c >= xc0;
                    const int xs = s1 ? xc1 : xc0, cs = s1 ? c - xc0 : c;
                    const __nv_bfloat16 *row =
                        gy < P.H ? (s1 ? P.x1 : P.x0) + act_idx(b, gy, cs, 0, P.H, P.W, xs) * 8 : nullptr;
                    if (T9)
                        stage_plane(st + pl.xoff + (size_t)u * kZPlane, row, x0, kPx, P.W, &full[s]);
                    else
                        stage_plane(st + pl.xoff + (size_t)u * kXPlane, row, x0 - 1, kXPx, P.W, &full[s]);
                }
            }
        }
        // every copy issued has landed before the CTA may exit
        if (lane == 0)
            for (int s = 0; s < S && s < i; ++s)
                tc::mbar_wait(&full[s], (uint32_t)((i - s + S - 1) / S - 1) & 1u, kWaitIter);
    } else if (warp == 1) {
        // ---- MMA issue (one thread) ----
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16(kPx, N) | (1u << 15) | (1u << 16);   // A and B MN-major
            constexpr int kXStride = T9 ? kZPlane : kXPlane;
            int i = 0;
            for (; i < ntile; ++i) {
                const int s = i % S;
                if (!tc::mbar_wait(&full[s], (uint32_t)(i / S) & 1u, kWaitIter)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t sb = tc::smem_u32(smem + (size_t)s * stage_bytes);
                // descriptors of row 0, pixel group 0; rows, groups and taps
                // at constant strides (start field in 16-byte units)
                const uint64_t bd0 = tc::sdesc(sb + (uint32_t)pl.zoff, 128, kZPlane);
                const uint64_t ad0 = tc::sdesc(sb + (uint32_t)pl.xoff, 128, kXStride);
                for (int r = 0; r < R; ++r) {
                    const uint64_t br = bd0 + ((uint64_t)(r * kZRow * kZPlane) >> 4);
                    const uint64_t ar = ad0 + ((uint64_t)(r * xc * kXStride) >> 4);
#pragma unroll
                    for (int g = 0; g < kPx / 16; ++g) {
                        const uint32_t acc = (i | r | g) ? 1u : 0u;
                        const uint64_t bg = br + ((uint64_t)(256 * g) >> 4), ag = ar + ((uint64_t)(256 * g) >> 4);
                        if (T9) {
                            tc::mma_bf16(tbase, ag, bg, idesc, acc);
                        } else {
#pragma unroll
                            for (int kx = 0; kx < 3; ++kx) tc::mma_bf16(tbase + kx * N, ag + kx, bg, idesc, acc);
                        }
                    }
                }
                tc::commit(&empty[s]);
            }
            // the last MMAs are done before the accumulators are read
            if (ok && i >= 1) ok = tc::mbar_wait(&empty[(i - 1) % S], (uint32_t)((i - 1) / S) & 1u, kWaitIter);
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    } else {
        // ---- bias warps: the tile's centre gradient rows (staged rows 1..R;
        // the nine-tap form's unshifted copy kx = 1) ----
        const int px = tid - 64;
        for (int i = 0; i < ntile; ++i) {
            const int s = i % S;
            bool got = true;
            if (lane == 0) got = tc::mbar_wait(&full[s], (uint32_t)(i / S) & 1u, kWaitIter);
            if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) {
                ok = false;
                break;
            }
            const uint8_t *st = smem + (size_t)s * stage_bytes + pl.zoff;
            for (int r = 1; r <= R; ++r)
#pragma unroll
                for (int c = 0; c < ZC; ++c) {
                    const int plane = r * kZRow + (T9 ? ZC : 0) + c;
                    const uint4 raw = *reinterpret_cast<const uint4 *>(st + (size_t)plane * kZPlane + 16 * px);
                    const __nv_bfloat162 *h2 = reinterpret_cast<const __nv_bfloat162 *>(&raw);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float2 f = __bfloat1622float2(h2[e]);
                        bsum[8 * c + 2 * e] += f.x;
                        bsum[8 * c + 2 * e + 1] += f.y;
                    }
                }
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(&empty[s]))
                                        : "memory");
        }
    }
    ok = __syncthreads_and(ok) != 0;
    tc::fence_after_sync();
    float *out = P.partial + (size_t)blockIdx.x * (9 * P.cin * P.cout + P.cout);
    if (!ok) {
        if (tid == 0) atomicExch(P.err, 1);
    } else if (ntile >= 1 && warp >= 2) {
        const int bw = warp - 2;
        // bias: lanes, then the four warps in a fixed order
#pragma unroll
        for (int j = 0; j < 8 * ZC; ++j) {
            float v = bsum[j];
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[bw * 8 * ZC + j] = v;
        }
        asm volatile("bar.sync 1, %0;" ::"n"(kWgradBiasWarps * 32) : "memory");   // the bias warps only
        if (bw == 0 && lane < P.cout) {
            float v = 0.f;
            for (int w = 0; w < kWgradBiasWarps; ++w) v += red[w * 8 * ZC + lane];
            out[9 * P.cin * P.cout + lane] = v;
        }
        // TMEM lane m = input channel (chunks of source 0, then of source 1,
        // 8 channels each; the concatenation's channel index).  Column n of
        // MMA k: nine-tap form n = ((ky' * 3 + kx) * zc + chunk) * 8 + e,
        // three-tap form (MMA kx) n = (ky' * zc + chunk) * 8 + e, with
        // ky = 2 - ky' and output channel 8 chunk + e.
        const int q = warp & 3, m = q * 32 + lane;
        const bool valid = m < 8 * xc && m < P.cin;
#pragma unroll
        for (int k = 0; k < NMMA; ++k)
#pragma unroll
            for (int j = 0; j < N; j += 16) {
                float v[16];
                tc::tmem_ld16(tbase + ((uint32_t)(q * 32) << 16) + k * N + j, v);
                if (valid) {
#pragma unroll
                    for (int qq = 0; qq < 16; ++qq) {
                        const int n = j + qq, grp = n >> 3, tap = grp / ZC, co = 8 * (grp - tap * ZC) + (n & 7);
                        const int kyp = T9 ? tap / 3 : tap, kx = T9 ? tap - 3 * kyp : k;
                        if (kyp < 3 && co < P.cout) out[(((2 - kyp) * 3 + kx) * P.cin + m) * P.cout + co] = v[qq];
                    }
                }
            }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) tc::tmem_dealloc(tbase, cols);
}

template <int ZC, bool T9>
cudaError_t launch_wgrad3_t(const WgradParams &P, const Wgrad3Plan &p, int B, int grid, cudaStream_t st)
{
    if (p.S < 2) return cudaErrorInvalidValue;
    cudaError_t e =
        cudaFuncSetAttribute(wgrad3_kernel<ZC, T9>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
    if (e != cudaSuccess) return e;
    const int ntx = (P.W + kPx - 1) / kPx, nty = (P.H + p.R - 1) / p.R;
    wgrad3_kernel<ZC, T9><<<grid, kWgradThreads, p.smem, st>>>(P, p, ntx, nty, B * ntx * nty);
    return cudaGetLastError();
}

}  // namespace

// Output rows per CTA: 4 (more CTAs per SM than 8-row tiles; measured faster
// in the whole network although the row halo grows from 25 to 50 %).
constexpr int kConvRows = 4;
// Output rows per CTA of the ky-stacked form: its TMEM holds R + 4 row
// groups (two junk groups on each side), and its MMA count per output row
// falls with R ((R + 2) / R input rows per output row).
constexpr int kConvRowsStacked = 4;


// K-step table for input chunks split over two sources (c0 chunks of source
// 0, then c1 of source 1; 8 channels each), per source: channel pairs of
// every tap, then, for an odd last chunk, tap pairs (kx, kx+1) with the
// second half of (ky, 2, 3) unused.  half[h] = (ky, kx, chunk) with chunk the
// conv input chunk over both sources, or chunk -1.
int build_steps(int c0, int c1, KStep *steps, StepHalf (*half)[2])
{
    int n = 0;
    for (int src = 0; src < 2; ++src) {
        const int nc = src ? c1 : c0, g0 = src ? c0 : 0;
        for (int c = 0; c + 1 < nc; c += 2)
            for (int ky = 0; ky < 3; ++ky)
                for (int kx = 0; kx < 3; ++kx) {
                    steps[n] = KStep{ky, c * kPlane + kx * 16, kPlane, src};
                    half[n][0] = StepHalf{ky, kx, g0 + c};
                    half[n][1] = StepHalf{ky, kx, g0 + c + 1};
                    ++n;
                }
        if (nc & 1) {
            const int c = nc - 1;
            for (int ky = 0; ky < 3; ++ky)
                for (int kx = 0; kx < 3; kx += 2) {
                    steps[n] = KStep{ky, c * kPlane + kx * 16, 16, src};
                    half[n][0] = StepHalf{ky, kx, g0 + c};
                    half[n][1] = kx + 1 < 3 ? StepHalf{ky, kx + 1, g0 + c} : StepHalf{0, 0, -1};
                    ++n;
                }
        }
    }
    return n;
}

int build_steps_stacked(int c0, int c1, KStep *steps, StepHalf (*half)[2])
{
    int n = 0;
    for (int src = 0; src < 2; ++src) {
        const int nc = src ? c1 : c0, g0 = src ? c0 : 0;
        for (int c = 0; c + 1 < nc; c += 2)
            for (int kx = 0; kx < 3; ++kx) {
                steps[n] = KStep{0, c * kPlane + kx * 16, kPlane, src};
                half[n][0] = StepHalf{-1, kx, g0 + c};
                half[n][1] = StepHalf{-1, kx, g0 + c + 1};
                ++n;
            }
        if (nc & 1) {
            const int c = nc - 1;
            for (int kx = 0; kx < 3; kx += 2) {
                steps[n] = KStep{0, c * kPlane + kx * 16, 16, src};
                half[n][0] = StepHalf{-1, kx, g0 + c};
                half[n][1] = kx + 1 < 3 ? StepHalf{-1, kx + 1, g0 + c} : StepHalf{0, 0, -1};
                ++n;
            }
        }
    }
    return n;
}

namespace {
std::atomic<int> g_conv_stacked{1};
}
bool conv_stacked_enabled() { return g_conv_stacked.load(std::memory_order_relaxed) != 0; }
void set_conv_stacked(bool on) { g_conv_stacked.store(on ? 1 : 0, std::memory_order_relaxed); }

cudaError_t launch_conv3x3(const ConvParams &P, int B, int nout, cudaStream_t st)
{
    if (P.stacked) {
        constexpr int Rs = kConvRowsStacked;
        if (nout == 16 && tma::persistent_enabled() && pipe_steps_supported(P.nsteps)) {
            const ConvPipePlan p2 = conv_pipe_plan(P.nsteps, 3 * 16, P.c0, P.c1, Rs, kPipeSmem2);
            if (p2.S >= 2) return launch_pipe<16, Rs>(P, p2, 2, B, st);
            const ConvPipePlan p1 = conv_pipe_plan(P.nsteps, 3 * 16, P.c0, P.c1, Rs, kPipeSmem);
            if (p1.S >= 2) return launch_pipe<16, Rs>(P, p1, 1, B, st);
        }
        if (nout == 16) return launch_t<16, kConvRowsStacked, true>(P, B, st);
        if (nout == 32) return launch_t<32, kConvRowsStacked, true>(P, B, st);
        if (nout == 48) return launch_t<48, kConvRowsStacked, true>(P, B, st);
        return cudaErrorInvalidValue;
    }
    if (nout == 16) return launch_t<16, kConvRows, false>(P, B, st);
    if (nout == 32) return launch_rows<32, kConvRows>(P, B, st);
    if (nout == 48) return launch_rows<48, kConvRows>(P, B, st);
    return cudaErrorInvalidValue;
}

}  // namespace unet
}  // namespace cd

namespace cd {
namespace unet {

cudaError_t launch_pack_jobs(const PackJobs &J, cudaStream_t st)
{
    if (J.n < 1 || J.n > kMaxPackJobs) return cudaErrorInvalidValue;
    int most = 0;
    for (int j = 0; j < J.n; ++j) {
        const int n = J.job[j].T.nsteps * 2 * J.job[j].T.nout * (J.job[j].T.stacked ? 3 : 1) * 8;
        most = n > most ? n : most;
    }
    pack_jobs_kernel<<<dim3((most + 255) / 256, J.n), 256, 0, st>>>(J);
    return cudaGetLastError();
}

cudaError_t launch_pack(const float *w, __nv_bfloat16 *dst, const PackTable &T, cudaStream_t st)
{
    const int n = T.nsteps * 2 * T.nout * (T.stacked ? 3 : 1) * 8;
    pack_kernel<<<(n + 255) / 256, 256, 0, st>>>(w, dst, T);
    return cudaGetLastError();
}

size_t wgrad_tiles(int B, int H, int W) { return (size_t)B * ((W + kPx - 1) / kPx) * ((H + kWgradRows - 1) / kWgradRows); }


static int sm_count()
{
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

// The persistent kernel takes every layer whose (ky, cout) fit N
// (zc <= 4) and whose input channels fit M (at most 16 chunks).  The
// nine-tap form runs layers of one output-gradient chunk (N = 80 against
// three MMAs of N = 32: 60 against 89 us at 1920x1080); at two chunks its
// N = 144 MMAs measured slower than three of N = 48 (44 against 34 us at
// 960x540), so wider layers take the three-tap form.
static bool wgrad3_t9(const WgradParams &P) { return P.zc == 1; }

static Wgrad3Plan wgrad3_plan_of(const WgradParams &P) { return wgrad3_plan(P.xc0 + P.xc1, P.zc, wgrad3_t9(P)); }

static bool wgrad3_fits(const WgradParams &P)
{
    const int xc = P.xc0 + P.xc1;
    return P.zc >= 1 && P.zc <= 4 && xc >= 1 && xc <= 16 && wgrad3_plan_of(P).S >= 2;
}

// Partial-sum rows the weight gradient of this layer writes: one per CTA of
// the persistent kernel, one per tile otherwise.
int wgrad_partial_rows(const WgradParams &P, int B)
{
    if (!wgrad3_fits(P)) return (int)wgrad_tiles(B, P.H, P.W);
    const Wgrad3Plan p = wgrad3_plan_of(P);
    const int tiles = B * ((P.W + kPx - 1) / kPx) * ((P.H + p.R - 1) / p.R);
    return tiles < sm_count() ? tiles : sm_count();
}

size_t wgrad_partial_floats(int B, int H, int W, int cin, int cout)
{
    const size_t t = wgrad_tiles(B, H, W);
    return reduce_floats(9 * cin * cout + cout, (int)(t > 1024 ? t : 1024));
}

cudaError_t launch_wgrad(const WgradParams &P, int B, cudaStream_t st)
{
    if (P.cout > 32) return cudaErrorInvalidValue;
    if (wgrad3_fits(P)) {
        const int grid = wgrad_partial_rows(P, B);
        const Wgrad3Plan p = wgrad3_plan_of(P);
        switch (P.zc) {
        case 1: return launch_wgrad3_t<1, true>(P, p, B, grid, st);
        case 2: return launch_wgrad3_t<2, false>(P, p, B, grid, st);
        case 3: return launch_wgrad3_t<3, false>(P, p, B, grid, st);
        default: return launch_wgrad3_t<4, false>(P, p, B, grid, st);
        }
    }
    return P.cout <= 16 ? launch_wgrad_t<16>(P, B, st) : launch_wgrad_t<32>(P, B, st);
}

}  // namespace unet
}  // namespace cd

