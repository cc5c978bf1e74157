"""The tensor-core U-Net (cd_unet_* and cd_adam_update) against the PyTorch
restatement oracle/unet_torch.py.

Both forms of the 3x3 convolution kernels (ky-stacked MMAs, the default,
and one MMA per output row and tap) are checked layer by layer and for the
whole network, and the persistent ky-stacked kernel against the
one-tile-per-CTA one (bit-identical).

Tolerances (bf16 operands and stored activations, fp32 accumulation):
  single layer vs the same bf16-rounded operands in fp32:
      max |y - ref| <= 1e-2 * max |ref|   (one bf16 rounding of the output)
  weight gradients of a single layer (fp32 sums over all pixels):
      max |g - ref| <= 2e-3 * max |ref|
  whole network, forward, on 1/band = p^2 + 1e-4 and alpha:
      vs the bf16-emulating restatement (fp32): max err <= 1e-2 * max |ref|
      vs float64 (no bf16):                     max err <= 3e-2 * max |ref|
  whole-network parameter gradients, with the head's band bias at 1 so that
  band = 1 / (p^2 + 1e-4) is well conditioned (near p = 0 its derivative
  reaches ~1e6 and bf16 activations alone move the gradient by O(1)):
      vs autograd of the bf16-emulating restatement: per tensor
          max |g - ref| <= 3e-2 * max |ref|          (measured <= 1e-2)
      vs autograd in float64: cosine of the whole gradient >= 0.98
          (bf16 activations alone, in the emulation as on the GPU, move
          single quarter-resolution entries by up to ~30% of their max)
  Adam vs the Keras update in float64: rtol 1e-5.
"""
import numpy as np
import pytest
import torch

from gpu_util import N
from oracle import unet_torch as ut

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
LAYER_SHAPES = [(15, 8), (8, 8), (8, 16), (16, 16), (16, 32), (32, 32), (48, 16), (24, 8)]


def bf16(t):
    return t.to(torch.bfloat16).to(torch.float32)


def rand_act(B, H, W, C, g, pad=True):
    Cs = (C + 7) // 8 * 8 if pad else C
    x = torch.zeros((B, H, W, Cs))
    x[..., :C] = torch.randn((B, H, W, C), generator=g).abs()
    return x


def weights(cin, cout, g):
    lim = (6.0 / (9 * cin + 9 * cout)) ** 0.5
    return (torch.rand((3, 3, cin, cout), generator=g) * 2 - 1) * lim, torch.randn((cout,), generator=g) * 0.1


def close_to_max(got, ref, frac, what):
    err = (got - ref).abs().max().item()
    m = ref.abs().max().item()
    assert err <= frac * m, f"{what}: max err {err:.4g} > {frac} * max|ref| {m:.4g}"


@pytest.fixture(params=[1, 0], ids=["ky_stacked", "per_row"])
def conv_form(request, cd):
    """Both forms of the 3x3 convolution kernels (cd_set_unet_conv_stacked)."""
    L = cd._lib.lib()
    L.cd_set_unet_conv_stacked(request.param)
    yield request.param
    L.cd_set_unet_conv_stacked(1)


@pytest.mark.parametrize("cin,cout", LAYER_SHAPES)
def test_conv3x3_forward(cd, cuda, conv_form, cin, cout):
    g = torch.Generator().manual_seed(cin * 100 + cout)
    B, H, W = 2, 21, 150                       # partial tiles in x and y
    x = bf16(rand_act(B, H, W, cin, g))
    w, b = weights(cin, cout, g)
    y, ws = cd.unet.conv3x3(w.to(DEV), b.to(DEV), x.to(DEV, torch.bfloat16), cin, cout)
    torch.cuda.synchronize()
    assert ws[:4].view(torch.int32).item() == 0
    ref = ut.conv3x3(x[..., :cin].permute(0, 3, 1, 2), bf16(w), b).permute(0, 2, 3, 1)
    close_to_max(y[..., :cout].float().cpu(), ref, 1e-2, f"conv {cin}->{cout}")


@pytest.mark.parametrize("cin,cout", LAYER_SHAPES)
def test_conv3x3_dgrad(cd, cuda, conv_form, cin, cout):
    g = torch.Generator().manual_seed(cin * 10 + cout)
    B, H, W = 1, 18, 140
    dz = bf16(torch.randn((B, H, W, (cout + 7) // 8 * 8), generator=g))
    dz[..., cout:] = 0
    w, _ = weights(cin, cout, g)
    y, ws = cd.unet.conv3x3(w.to(DEV), None, dz.to(DEV, torch.bfloat16), cin, cout, dgrad=True)
    torch.cuda.synchronize()
    x = torch.zeros((B, cin, H, W), requires_grad=True)
    out = ut.conv3x3(x, bf16(w), None, relu=False)
    out.backward(dz[..., :cout].permute(0, 3, 1, 2))
    ref = x.grad.permute(0, 2, 3, 1)
    close_to_max(y[..., :cin].float().cpu(), ref, 1e-2, f"dgrad {cin}->{cout}")


@pytest.mark.parametrize("cin,cout", LAYER_SHAPES)
def test_conv3x3_wgrad(cd, cuda, cin, cout):
    g = torch.Generator().manual_seed(cin + cout * 7)
    B, H, W = 2, 19, 133
    x = bf16(rand_act(B, H, W, cin, g))
    dz = bf16(torch.randn((B, H, W, (cout + 7) // 8 * 8), generator=g))
    dz[..., cout:] = 0
    dW, db, ws = cd.unet.conv3x3_wgrad(x.to(DEV, torch.bfloat16), dz.to(DEV, torch.bfloat16), cin, cout)
    torch.cuda.synchronize()
    assert ws[:4].view(torch.int32).item() == 0
    K = torch.zeros((3, 3, cin, cout), requires_grad=True)
    bb = torch.zeros((cout,), requires_grad=True)
    out = ut.conv3x3(x[..., :cin].permute(0, 3, 1, 2).double(), K.double(), bb.double(), relu=False)
    out.backward(dz[..., :cout].permute(0, 3, 1, 2).double())
    close_to_max(dW.cpu(), K.grad.float(), 2e-3, f"wgrad {cin}->{cout}")
    close_to_max(db.cpu(), bb.grad.float(), 2e-3, f"bgrad {cin}->{cout}")


@pytest.mark.parametrize("cin,cout", [(8, 8), (15, 8), (32, 32), (48, 16)])
def test_conv3x3_wgrad_many_tiles(cd, cuda, cin, cout):
    """Enough tiles (2 x 512 x 1000) that every persistent CTA runs several
    and the staging ring wraps around more than once."""
    g = torch.Generator().manual_seed(cin * 3 + cout)
    B, H, W = 2, 512, 1000
    x = bf16(rand_act(B, H, W, cin, g))
    dz = bf16(torch.randn((B, H, W, (cout + 7) // 8 * 8), generator=g))
    dz[..., cout:] = 0
    dW, db, ws = cd.unet.conv3x3_wgrad(x.to(DEV, torch.bfloat16), dz.to(DEV, torch.bfloat16), cin, cout)
    torch.cuda.synchronize()
    assert ws[:4].view(torch.int32).item() == 0
    K = torch.zeros((3, 3, cin, cout), requires_grad=True)
    bb = torch.zeros((cout,), requires_grad=True)
    out = ut.conv3x3(x[..., :cin].permute(0, 3, 1, 2).double(), K.double(), bb.double(), relu=False)
    out.backward(dz[..., :cout].permute(0, 3, 1, 2).double())
    close_to_max(dW.cpu(), K.grad.float(), 2e-3, f"wgrad {cin}->{cout}")
    close_to_max(db.cpu(), bb.grad.float(), 2e-3, f"bgrad {cin}->{cout}")


def frame_inputs(B, H, W, seed):
    g = torch.Generator().manual_seed(seed)
    ols1 = torch.rand((B, H, W, 3), generator=g) * 3
    ols2 = ols1 + 0.2 * torch.randn((B, H, W, 3), generator=g)
    prev = ols1 * 0.9
    alb = torch.rand((B, H, W, 3), generator=g)
    n = torch.randn((B, H, W, 3), generator=g)
    nrm = n / n.norm(dim=-1, keepdim=True)
    return [ols1, ols2, prev, alb, nrm]


def reference(params, ins, bf16_emulation, gb=None, ga=None):
    dt = torch.float32 if bf16_emulation else torch.float64
    p = params.cpu().clone().to(dt).requires_grad_(gb is not None)
    band, alpha = ut.forward(p, *[t.to(dt) for t in ins], bf16=bf16_emulation)
    if gb is None:
        return band.double(), alpha.double()
    ((band * gb.to(dt)).sum() + (alpha * ga.to(dt)).sum()).backward()
    return p.grad.double()


def test_unet_forward(cd, cuda, conv_form):
    B, H, W = 1, 36, 264
    ins = frame_inputs(B, H, W, 5)
    net = cd.unet.UNet(DEV, seed=3)
    band, alpha = net(*[t.to(DEV) for t in ins])
    torch.cuda.synchronize()
    assert net.error_flag() == 0
    for emu, tol in ((True, 1e-2), (False, 3e-2)):
        rb, ra = reference(net.params, ins, emu)
        close_to_max(1.0 / band.cpu().double(), 1.0 / rb, tol, f"1/band (bf16 emulation {emu})")
        close_to_max(alpha.cpu().double(), ra, tol, f"alpha (bf16 emulation {emu})")


def well_conditioned_net(cd, seed):
    p = cd.unet.glorot_init(seed)
    parts = cd.unet.split_params(p)
    parts[-1][:5] = 1.0        # head bias of the five band channels: p near 1
    return cd.unet.UNet(DEV, params=p)


def test_unet_backward_and_adam(cd, cuda, conv_form):
    B, H, W = 1, 64, 264
    ins = frame_inputs(B, H, W, 7)
    net = well_conditioned_net(cd, 4)
    g = torch.Generator().manual_seed(8)
    gb = torch.randn((B, H, W, 5), generator=g)
    ga = torch.randn((B, H, W, 1), generator=g)
    net(*[t.to(DEV) for t in ins])
    grads = net.backward(gb.to(DEV), ga.to(DEV)).cpu().clone().double()
    torch.cuda.synchronize()
    assert net.error_flag() == 0
    ref = reference(net.params, ins, True, gb, ga)
    o = 0
    for i, shape in enumerate(cd.unet.param_shapes()):
        n = int(np.prod(shape))
        close_to_max(grads[o:o + n], ref[o:o + n], 3e-2, f"param tensor {i} {shape}")
        o += n
    ref64 = reference(net.params, ins, False, gb, ga)
    cos = (grads @ ref64 / (grads.norm() * ref64.norm())).item()
    assert cos >= 0.98, f"gradient direction vs float64: cosine {cos:.4f}"
    # Adam: three Keras updates in float64 vs cd_adam_update
    w64 = net.params.cpu().double().clone()
    m64, v64 = torch.zeros_like(w64), torch.zeros_like(w64)
    for step in range(1, 4):
        ut.adam_keras(w64, grads, m64, v64, step)
        net.apply_gradients()
    torch.cuda.synchronize()
    np.testing.assert_allclose(N(net.params), w64.numpy(), rtol=1e-5, atol=1e-7)


def test_persistent_conv_matches_per_tile(cd, cuda):
    """The persistent warp-specialised convolution (16-output layers) issues
    the one-tile-per-CTA kernel's MMAs in the same order into the same
    accumulator layout: forward outputs and every parameter gradient are
    bit-identical with the persistent kernels on and off, at a shape with
    ragged tiles (H not a multiple of 4 rows at every level, W of 128)."""
    L = cd._lib.lib()
    B, H, W = 2, 76, 392
    ins = [t.to(DEV) for t in frame_inputs(B, H, W, 11)]
    g = torch.Generator().manual_seed(12)
    gb = torch.randn((B, H, W, 5), generator=g).to(DEV)
    ga = torch.randn((B, H, W, 1), generator=g).to(DEV)
    out = {}
    try:
        for on in (1, 0):
            L.cd_set_persistent_kernels(on)
            net = well_conditioned_net(cd, 9)
            band, alpha = net(*ins)
            grads = net.backward(gb, ga)
            torch.cuda.synchronize()
            assert net.error_flag() == 0
            out[on] = (band.clone(), alpha.clone(), grads.clone())
    finally:
        L.cd_set_persistent_kernels(1)
    for a, b, what in zip(out[1], out[0], ("band", "alpha", "parameter gradients")):
        assert torch.equal(a, b), f"{what} differ between the persistent and per-tile convolutions"


def test_shape_errors(cd, cuda):
    net = cd.unet.UNet(DEV)
    x = torch.zeros((1, 30, 64, 3), device=DEV)
    with pytest.raises(ValueError):
        net(x, x, x, x, x)
