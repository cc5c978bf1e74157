// The reference's kernel-predicting U-Net (scripts/main.py:83-118) on the
// tensor cores: forward, backward and the Adam update, orchestrated here on
// the host side of the C ABI.
//
// Layers (Keras trainable-variable order; parameters are one flat fp32
// buffer, each layer's kernel in Keras layout followed by its bias):
//   L0  conv 15->8   full        L6  tconv 32->32  quarter->half
//   L1  conv 8->8    full (+pool) L7  conv 48->16   half  (in: L6 | L3)
//   L2  conv 8->16   half        L8  conv 16->16   half
//   L3  conv 16->16  half (+pool) L9  tconv 16->16  half->full
//   L4  conv 16->32  quarter     L10 conv 24->8    full  (in: L9 | L1)
//   L5  conv 32->32  quarter     L11 head 8->6 (1x1, fp32) -> band, alpha
// 31,414 parameters.  Activations and activation gradients are bf16
// row-chunk planes (unet.cuh) in the workspace; the forward keeps every
// activation for the backward.
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "cd_common.cuh"
#include "unet.cuh"
#include "unet_ops.cuh"

namespace cd {
namespace unet {
namespace {

enum Kind { CONV, TCONV, HEAD };
struct LayerDef {
    Kind kind;
    int cin, cout;
};
constexpr int kLayers = 12;
constexpr LayerDef kDef[kLayers] = {{CONV, 15, 8},   {CONV, 8, 8},    {CONV, 8, 16},  {CONV, 16, 16},
                                    {CONV, 16, 32},  {CONV, 32, 32},  {TCONV, 32, 32}, {CONV, 48, 16},
                                    {CONV, 16, 16},  {TCONV, 16, 16}, {CONV, 24, 8},  {HEAD, 8, 6}};

int param_size(const LayerDef &d)
{
    return d.kind == CONV ? 9 * d.cin * d.cout + d.cout : d.cin * d.cout + d.cout;
}
int param_offset(int l)
{
    int o = 0;
    for (int i = 0; i < l; ++i) o += param_size(kDef[i]);
    return o;
}
int weight_count(int l) { return param_size(kDef[l]) - kDef[l].cout; }
int chunks(int c) { return (c + 7) / 8; }
int nout_of(int c) { return c <= 16 ? 16 : (c <= 32 ? 32 : 48); }

// activation / gradient tensors: channels and pyramid level
enum Buf {
    X0, C11, C12, C13, C21, C22, C23, C31, C32, C33, C41, C42, C43, C51,
    DZ10, DC43, DSK1, DZ8, DZ7, DC33, DSK2, DZ5, DZ4, DC23, DZ3, DZ2, DC13, DZ1, DZ0, NBUF
};
constexpr int kBufCh[NBUF] = {16, 8, 8, 8, 16, 16, 16, 32, 32, 32, 16, 16, 16, 8,
                              8, 16, 8, 16, 16, 32, 16, 32, 32, 16, 16, 16, 8, 8, 8};
constexpr int kBufLvl[NBUF] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 1, 1, 1, 0, 0,
                               0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 0, 0};

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Workspace: [error flag][packed weights per conv: fwd, dgrad][buffers][partials]
struct Layout {
    size_t pack_fwd[kLayers], pack_dg[kLayers], buf[NBUF], partial, partial2, total;
    int steps_fwd[kLayers], steps_dg[kLayers];
};

// forward input split over the two sources of a concatenation (chunks of 8
// channels): L7 reads [c3_3 | c2_2], L10 reads [c4_3 | c1_2]
constexpr int kSrc0[kLayers] = {2, 1, 1, 2, 2, 4, 0, 4, 2, 0, 2, 0};
constexpr int kSrc1[kLayers] = {0, 0, 0, 0, 0, 0, 0, 2, 0, 0, 1, 0};

// pyramid level of each layer's input (0 full, 1 half, 2 quarter)
constexpr int kLvl[kLayers] = {0, 0, 1, 1, 2, 2, 2, 1, 1, 1, 0, 0};

size_t partial_floats(int B, int H, int W)
{
    size_t m = 0;
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef &d = kDef[l];
        const int h = H >> kLvl[l], w = W >> kLvl[l];
        size_t n = 0;
        if (d.kind == CONV) n = wgrad_partial_floats(B, h, w, d.cin, d.cout);
        else if (d.kind == TCONV) n = reduce_floats(d.cin * d.cout + d.cout, (int)tconv_blocks(d.cin, h, w, B));
        else n = reduce_floats(54, (int)head_blocks((size_t)B * H * W));
        m = n > m ? n : m;
    }
    return m;
}

Layout layout(int B, int H, int W)
{
    Layout L{};
    size_t o = 256;   // error flag
    KStep st[kMaxSteps];
    StepHalf hf[kMaxSteps][2];
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef &d = kDef[l];
        if (d.kind != CONV) continue;
        L.steps_fwd[l] = build_steps(kSrc0[l], kSrc1[l], st, hf);
        L.pack_fwd[l] = o;
        o += align256((size_t)L.steps_fwd[l] * 2 * nout_of(d.cout) * 16);
        L.steps_dg[l] = build_steps(chunks(d.cout), 0, st, hf);
        L.pack_dg[l] = o;
        o += align256((size_t)L.steps_dg[l] * 2 * nout_of(d.cin) * 16);
    }
    for (int i = 0; i < NBUF; ++i) {
        L.buf[i] = o;
        o += align256((size_t)B * (H >> kBufLvl[i]) * (W >> kBufLvl[i]) * kBufCh[i] * 2);
    }
    L.partial = o;
    o += align256(partial_floats(B, H, W) * sizeof(float));
    L.partial2 = o;   // the weight gradients' partials (companion stream)
    o += align256(partial_floats(B, H, W) * sizeof(float));
    L.total = o;
    return L;
}

struct Ctx {
    uint8_t *ws;
    Layout L;
    int B, H, W;
    cudaStream_t st;
    const float *params;
    bool stacked = conv_stacked_enabled();   // the convolution form of this call (packing and kernels agree)
    // the ky-stacked form where it measured faster: 16 conv output channels
    bool stacked_for(int nout) const { return stacked && nout == 16; }
    __nv_bfloat16 *buf(Buf b) const { return reinterpret_cast<__nv_bfloat16 *>(ws + L.buf[b]); }
    int *err() const { return reinterpret_cast<int *>(ws); }
    float *partial() const { return reinterpret_cast<float *>(ws + L.partial); }
    float *partial2() const { return reinterpret_cast<float *>(ws + L.partial2); }
    const float *w(int l) const { return params + param_offset(l); }
    const float *b(int l) const { return params + param_offset(l) + weight_count(l); }
};

#define CD_TRY(x)                          \
    do {                                   \
        cudaError_t e_ = (x);              \
        if (e_ != cudaSuccess) return e_;  \
    } while (0)

// Pack the B operands of every 3x3 layer (forward tables, or the dgrad
// tables of layers 1..10) in one launch.
cudaError_t pack_all(const Ctx &c, bool dgrad)
{
    PackJobs J{};
    for (int l = dgrad ? 1 : 0; l < kLayers; ++l) {
        const LayerDef &d = kDef[l];
        if (d.kind != CONV) continue;
        PackJob &j = J.job[J.n++];
        KStep st[kMaxSteps];
        const int nout = nout_of(dgrad ? d.cin : d.cout);
        auto steps = c.stacked_for(nout) ? build_steps_stacked : build_steps;
        j.T.nsteps = dgrad ? steps(chunks(d.cout), 0, st, j.T.half) : steps(kSrc0[l], kSrc1[l], st, j.T.half);
        j.T.stacked = c.stacked_for(nout) ? 1 : 0;
        j.T.nout = nout;
        j.T.cin = d.cin;
        j.T.cout = d.cout;
        j.T.dgrad = dgrad ? 1 : 0;
        j.w = c.w(l);
        j.dst = reinterpret_cast<__nv_bfloat16 *>(c.ws + (dgrad ? c.L.pack_dg[l] : c.L.pack_fwd[l]));
    }
    return launch_pack_jobs(J, c.st);
}

// conv of `l` (forward, or dgrad when dgrad) at pyramid level lvl
cudaError_t conv(const Ctx &c, int l, bool dgrad, int lvl, Buf s0, int c0, Buf s1, int c1, Buf d0, int dc0, Buf d1,
                 int dc1, Buf m0, Buf m1, Buf pool)
{
    const LayerDef &d = kDef[l];
    ConvParams P{};
    StepHalf hf[kMaxSteps][2];
    const bool stacked = c.stacked_for(nout_of(dgrad ? d.cin : d.cout));
    P.nsteps = (stacked ? build_steps_stacked : build_steps)(c0, c1, P.steps, hf);
    P.stacked = stacked ? 1 : 0;
    P.src0 = c.buf(s0);
    P.src1 = c1 ? c.buf(s1) : nullptr;
    P.c0 = c0;
    P.c1 = c1;
    P.wpack = reinterpret_cast<const __nv_bfloat16 *>(c.ws + (dgrad ? c.L.pack_dg[l] : c.L.pack_fwd[l]));
    P.bias = dgrad ? nullptr : c.b(l);
    P.dst0 = c.buf(d0);
    P.dst1 = dc1 ? c.buf(d1) : nullptr;
    P.d0 = dc0;
    P.d1 = dc1;
    P.mask0 = m0 == NBUF ? nullptr : c.buf(m0);
    P.mask1 = m1 == NBUF ? nullptr : c.buf(m1);
    P.pool = pool == NBUF ? nullptr : c.buf(pool);
    P.relu = dgrad ? 0 : 1;
    P.H = c.H >> lvl;
    P.W = c.W >> lvl;
    P.err = c.err();
    return launch_conv3x3(P, c.B, nout_of(dgrad ? d.cin : d.cout), c.st);
}

// Weight and bias gradient of layer l on stream `st` with partial buffer `part`.
cudaError_t wgrad(const Ctx &c, float *grads, int l, int lvl, Buf x0, int xc0, Buf x1, int xc1, Buf dz,
                  cudaStream_t st, float *part)
{
    const LayerDef &d = kDef[l];
    WgradParams P{};
    P.x0 = c.buf(x0);
    P.x1 = xc1 ? c.buf(x1) : nullptr;
    P.xc0 = xc0;
    P.xc1 = xc1;
    P.dz = c.buf(dz);
    P.zc = chunks(d.cout);
    P.cin = d.cin;
    P.cout = d.cout;
    P.partial = part;
    P.H = c.H >> lvl;
    P.W = c.W >> lvl;
    P.err = c.err();
    CD_TRY(launch_wgrad(P, c.B, st));
    return launch_reduce(part, grads + param_offset(l), param_size(d), wgrad_partial_rows(P, c.B), st);
}

// A companion stream per caller stream (and device) for the weight
// gradients, which depend only on their layer's dZ and the forward
// activations: each is forked after the kernel that writes its dZ (event
// record / wait, which stream capture records as graph edges) and overlaps
// the rest of the input-gradient chain; backward() joins it before
// returning.  Companions are created on first use outside stream capture;
// inside a capture without one, the gradients stay on the caller's stream.
struct Side {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

Side *side_stream(cudaStream_t main)
{
    static std::mutex mu;
    static std::unordered_map<uint64_t, Side> sides;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    const uint64_t key = (reinterpret_cast<uint64_t>(main) << 8) ^ (uint64_t)dev;
    std::lock_guard<std::mutex> lock(mu);
    auto it = sides.find(key);
    if (it != sides.end()) return &it->second;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(main, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    Side sd;
    int prio = 0;   // the companion runs at the caller's stream priority
    if (cudaStreamGetPriority(main, &prio) != cudaSuccess) prio = 0;
    if (cudaStreamCreateWithPriority(&sd.s, cudaStreamNonBlocking, prio) != cudaSuccess) return nullptr;
    if (cudaEventCreateWithFlags(&sd.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sd.join, cudaEventDisableTiming) != cudaSuccess)
        return nullptr;
    return &(sides[key] = sd);
}

constexpr Buf NONE = NBUF;

}  // namespace

int param_count() { return param_offset(kLayers); }
size_t workspace_bytes(int B, int H, int W) { return layout(B, H, W).total; }

cudaError_t forward(const float *ols1, const float *ols2, const float *prev, const float *albedo,
                    const float *normal, const float *params, float *band, float *alpha, void *ws, int B, int H,
                    int W, cudaStream_t st)
{
    Ctx c{static_cast<uint8_t *>(ws), layout(B, H, W), B, H, W, st, params};
    const size_t n0 = (size_t)B * H * W;
    CD_TRY(pack_all(c, false));
    CD_TRY(launch_pack_input(ols1, ols2, prev, albedo, normal, c.buf(X0), n0, W, st));
    CD_TRY(conv(c, 0, false, 0, X0, 2, NONE, 0, C11, 1, NONE, 0, NONE, NONE, NONE));
    CD_TRY(conv(c, 1, false, 0, C11, 1, NONE, 0, C12, 1, NONE, 0, NONE, NONE, C13));
    CD_TRY(conv(c, 2, false, 1, C13, 1, NONE, 0, C21, 2, NONE, 0, NONE, NONE, NONE));
    CD_TRY(conv(c, 3, false, 1, C21, 2, NONE, 0, C22, 2, NONE, 0, NONE, NONE, C23));
    CD_TRY(conv(c, 4, false, 2, C23, 2, NONE, 0, C31, 4, NONE, 0, NONE, NONE, NONE));
    CD_TRY(conv(c, 5, false, 2, C31, 4, NONE, 0, C32, 4, NONE, 0, NONE, NONE, NONE));
    CD_TRY(launch_tconv_fwd(32, 32, c.buf(C32), c.w(6), c.b(6), c.buf(C33), H >> 2, W >> 2, B, st));
    CD_TRY(conv(c, 7, false, 1, C33, 4, C22, 2, C41, 2, NONE, 0, NONE, NONE, NONE));
    CD_TRY(conv(c, 8, false, 1, C41, 2, NONE, 0, C42, 2, NONE, 0, NONE, NONE, NONE));
    CD_TRY(launch_tconv_fwd(16, 16, c.buf(C42), c.w(9), c.b(9), c.buf(C43), H >> 1, W >> 1, B, st));
    CD_TRY(conv(c, 10, false, 0, C43, 2, C12, 1, C51, 1, NONE, 0, NONE, NONE, NONE));
    return launch_head_fwd(c.buf(C51), c.w(11), c.b(11), band, alpha, n0, st);
}

cudaError_t backward(const float *gband, const float *galpha, const float *params, float *grads, void *ws, int B,
                     int H, int W, cudaStream_t st)
{
    Ctx c{static_cast<uint8_t *>(ws), layout(B, H, W), B, H, W, st, params};
    const size_t n0 = (size_t)B * H * W;
    Side *side = side_stream(st);
    // weight gradient of layer l, forked onto the companion stream when there is one
    auto wg = [&](int l, int lvl, Buf x0, int xc0, Buf x1, int xc1, Buf dz) -> cudaError_t {
        if (!side) return wgrad(c, grads, l, lvl, x0, xc0, x1, xc1, dz, st, c.partial2());
        CD_TRY(cudaEventRecord(side->fork, st));
        CD_TRY(cudaStreamWaitEvent(side->s, side->fork, 0));
        return wgrad(c, grads, l, lvl, x0, xc0, x1, xc1, dz, side->s, c.partial2());
    };
    auto body = [&]() -> cudaError_t {
        CD_TRY(pack_all(c, true));
        // head
        CD_TRY(launch_head_bwd(c.buf(C51), c.w(11), c.b(11), gband, galpha, c.buf(DZ10), c.partial(), n0, st));
        CD_TRY(launch_reduce(c.partial(), grads + param_offset(11), 54, (int)head_blocks(n0), st));
        // L10: 24 -> 8 at full resolution; input gradient splits into c4_3 and the c1_2 skip
        CD_TRY(wg(10, 0, C43, 2, C12, 1, DZ10));
        CD_TRY(conv(c, 10, true, 0, DZ10, 1, NONE, 0, DC43, 2, DSK1, 1, NONE, NONE, NONE));
        // L9: transposed conv half -> full
        CD_TRY(launch_tconv_bwd(16, 16, c.buf(C42), c.buf(DC43), c.w(9), c.buf(DZ8), c.partial(), H >> 1, W >> 1, B,
                                st));
        CD_TRY(launch_reduce(c.partial(), grads + param_offset(9), param_size(kDef[9]),
                             (int)tconv_blocks(16, H >> 1, W >> 1, B), st));
        // L8
        CD_TRY(wg(8, 1, C41, 2, NONE, 0, DZ8));
        CD_TRY(conv(c, 8, true, 1, DZ8, 2, NONE, 0, DZ7, 2, NONE, 0, C41, NONE, NONE));
        // L7: 48 -> 16; input gradient splits into c3_3 and the c2_2 skip
        CD_TRY(wg(7, 1, C33, 4, C22, 2, DZ7));
        CD_TRY(conv(c, 7, true, 1, DZ7, 2, NONE, 0, DC33, 4, DSK2, 2, NONE, NONE, NONE));
        // L6: transposed conv quarter -> half
        CD_TRY(launch_tconv_bwd(32, 32, c.buf(C32), c.buf(DC33), c.w(6), c.buf(DZ5), c.partial(), H >> 2, W >> 2, B,
                                st));
        CD_TRY(launch_reduce(c.partial(), grads + param_offset(6), param_size(kDef[6]),
                             (int)tconv_blocks(32, H >> 2, W >> 2, B), st));
        // L5, L4
        CD_TRY(wg(5, 2, C31, 4, NONE, 0, DZ5));
        CD_TRY(conv(c, 5, true, 2, DZ5, 4, NONE, 0, DZ4, 4, NONE, 0, C31, NONE, NONE));
        CD_TRY(wg(4, 2, C23, 2, NONE, 0, DZ4));
        CD_TRY(conv(c, 4, true, 2, DZ4, 4, NONE, 0, DC23, 2, NONE, 0, NONE, NONE, NONE));
        // pool of c2_2 + skip, ReLU of c2_2
        CD_TRY(launch_pool_bwd(16, c.buf(C22), c.buf(C23), c.buf(DC23), c.buf(DSK2), c.buf(DZ3), H >> 1, W >> 1, B,
                               st));
        // L3, L2
        CD_TRY(wg(3, 1, C21, 2, NONE, 0, DZ3));
        CD_TRY(conv(c, 3, true, 1, DZ3, 2, NONE, 0, DZ2, 2, NONE, 0, C21, NONE, NONE));
        CD_TRY(wg(2, 1, C13, 1, NONE, 0, DZ2));
        CD_TRY(conv(c, 2, true, 1, DZ2, 2, NONE, 0, DC13, 1, NONE, 0, NONE, NONE, NONE));
        // pool of c1_2 + skip, ReLU of c1_2
        CD_TRY(launch_pool_bwd(8, c.buf(C12), c.buf(C13), c.buf(DC13), c.buf(DSK1), c.buf(DZ1), H, W, B, st));
        // L1, L0
        CD_TRY(wg(1, 0, C11, 1, NONE, 0, DZ1));
        CD_TRY(conv(c, 1, true, 0, DZ1, 1, NONE, 0, DZ0, 1, NONE, 0, C11, NONE, NONE));
        return wg(0, 0, X0, 2, NONE, 0, DZ0);
    };
    const cudaError_t e = body();
    if (side) {   // join, also after a failed launch, so no fork is left open
        const cudaError_t e1 = cudaEventRecord(side->join, side->s);
        const cudaError_t e2 = cudaStreamWaitEvent(st, side->join, 0);
        if (e == cudaSuccess && e1 != cudaSuccess) return e1;
        if (e == cudaSuccess && e2 != cudaSuccess) return e2;
    }
    return e;
}

size_t conv_layer_workspace(int cin, int cout)
{
    KStep st[kMaxSteps];
    StepHalf hf[kMaxSteps][2];
    const int a = build_steps(chunks(cin), 0, st, hf), b = build_steps(chunks(cout), 0, st, hf);
    const size_t fw = (size_t)a * 2 * nout_of(cout) * 16, dg = (size_t)b * 2 * nout_of(cin) * 16;
    return 256 + align256(fw > dg ? fw : dg);
}

cudaError_t conv_layer(const float *w, const float *bias, const __nv_bfloat16 *x, __nv_bfloat16 *y, int cin,
                       int cout, int dgrad, int B, int H, int W, void *ws, cudaStream_t st)
{
    uint8_t *base = static_cast<uint8_t *>(ws);
    __nv_bfloat16 *wp = reinterpret_cast<__nv_bfloat16 *>(base + 256);
    const int in_ch = dgrad ? cout : cin, out_ch = dgrad ? cin : cout;
    const bool stacked = conv_stacked_enabled() && nout_of(out_ch) == 16;   // as Ctx::stacked_for
    auto steps = stacked ? build_steps_stacked : build_steps;
    PackTable T{};
    KStep st_[kMaxSteps];
    T.nsteps = steps(chunks(in_ch), 0, st_, T.half);
    T.nout = nout_of(out_ch);
    T.cin = cin;
    T.cout = cout;
    T.dgrad = dgrad;
    T.stacked = stacked ? 1 : 0;
    CD_TRY(launch_pack(w, wp, T, st));
    ConvParams P{};
    StepHalf hf[kMaxSteps][2];
    P.nsteps = steps(chunks(in_ch), 0, P.steps, hf);
    P.stacked = stacked ? 1 : 0;
    P.src0 = x;
    P.c0 = chunks(in_ch);
    P.wpack = wp;
    P.bias = dgrad ? nullptr : bias;
    P.dst0 = y;
    P.d0 = chunks(out_ch);
    P.relu = dgrad ? 0 : 1;
    P.H = H;
    P.W = W;
    P.err = reinterpret_cast<int *>(base);
    return launch_conv3x3(P, B, T.nout, st);
}

size_t wgrad_layer_workspace(int cin, int cout, int B, int H, int W)
{
    return 256 + align256(wgrad_partial_floats(B, H, W, cin, cout) * sizeof(float));
}

cudaError_t wgrad_layer(const __nv_bfloat16 *x, const __nv_bfloat16 *dz, float *grad, int cin, int cout, int B,
                        int H, int W, void *ws, cudaStream_t st)
{
    uint8_t *base = static_cast<uint8_t *>(ws);
    WgradParams P{};
    P.x0 = x;
    P.xc0 = chunks(cin);
    P.dz = dz;
    P.zc = chunks(cout);
    P.cin = cin;
    P.cout = cout;
    P.partial = reinterpret_cast<float *>(base + 256);
    P.H = H;
    P.W = W;
    P.err = reinterpret_cast<int *>(base);
    CD_TRY(launch_wgrad(P, B, st));
    return launch_reduce(P.partial, grad, 9 * cin * cout + cout, wgrad_partial_rows(P, B), st);
}

cudaError_t adam(float *w, const float *g, float *m, float *v, int n, int *step, float lr, float b1, float b2,
                 float eps, cudaStream_t st)
{
    return launch_adam(w, g, m, v, n, step, lr, b1, b2, eps, st);
}

}  // namespace unet
}  // namespace cd
