"""Host-side pieces of the U-Net (no GPU): the parameter layout of the
reference's model (scripts/main.py:83-108; 31,414 parameters), the Keras
initialiser, and the PyTorch restatement used as the GPU oracle."""
import numpy as np
import torch

from oracle import unet_torch as ut


def test_param_layout(cd):
    shapes = cd.unet.param_shapes()
    assert len(shapes) == 24
    assert cd.unet.param_count() == 31414
    # conv kernels (3,3,cin,cout); transposed convs (1,1,cout,cin); head (1,1,8,6)
    assert shapes[0] == (3, 3, 15, 8) and shapes[12] == (1, 1, 32, 32) and shapes[22] == (1, 1, 8, 6)
    assert [s for s in shapes[1::2]] == [(c,) for _, _, c in cd.unet.LAYERS]


def test_glorot_init(cd):
    p = cd.unet.glorot_init(7)
    assert p.dtype == np.float32 and p.size == 31414
    np.testing.assert_array_equal(p, cd.unet.glorot_init(7))
    for t, shape in zip(cd.unet.split_params(p), cd.unet.param_shapes()):
        if len(shape) == 1:
            assert not t.any()
        else:
            rf = shape[0] * shape[1]
            lim = np.sqrt(6.0 / (shape[2] * rf + shape[3] * rf))
            assert np.abs(t).max() <= lim
            assert np.abs(t).max() > 0.8 * lim


def test_transposed_conv_places_even_positions():
    g = torch.Generator().manual_seed(0)
    x = torch.randn((1, 4, 3, 5), generator=g, dtype=torch.float64)
    K = torch.randn((1, 1, 6, 4), generator=g, dtype=torch.float64)
    b = torch.randn((6,), generator=g, dtype=torch.float64)
    y = ut.tconv(x, K, b)
    assert y.shape == (1, 6, 6, 10)
    want = torch.einsum("oc,bchw->bohw", K[0, 0], x) + b.view(1, -1, 1, 1)
    torch.testing.assert_close(y[:, :, 0::2, 0::2], want)
    for sl in ((slice(1, None, 2), slice(None)), (slice(None), slice(1, None, 2))):
        torch.testing.assert_close(y[:, :, sl[0], sl[1]], b.view(1, -1, 1, 1).expand_as(y[:, :, sl[0], sl[1]]))


def test_forward_shapes_and_ranges(cd):
    B, H, W = 2, 8, 12
    g = torch.Generator().manual_seed(1)
    ins = [torch.rand((B, H, W, 3), generator=g, dtype=torch.float64) for _ in range(5)]
    p = torch.from_numpy(cd.unet.glorot_init(3)).double()
    keep = {}
    band, alpha = ut.forward(p, *ins, keep=keep)
    assert band.shape == (B, H, W, 5) and alpha.shape == (B, H, W, 1)
    assert (band > 0).all() and (band <= 1e4 + 1e-6).all()
    assert ((alpha > 0) & (alpha < 1)).all()
    assert keep["c13"].shape == (B, 8, H // 2, W // 2) and keep["c33"].shape == (B, 32, H // 2, W // 2)
    # bf16 emulation stays close to the exact network
    b2, a2 = ut.forward(p.float(), *[t.float() for t in ins], bf16=True)
    assert (1 / b2.double() - 1 / band).abs().max() < 3e-2 * (1 / band).abs().max()


def test_adam_matches_closed_form():
    p = torch.tensor([1.0, -2.0], dtype=torch.float64)
    m, v = torch.zeros(2, dtype=torch.float64), torch.zeros(2, dtype=torch.float64)
    g = torch.tensor([0.5, -0.25], dtype=torch.float64)
    ut.adam_keras(p, g, m, v, 1)
    # first step: m = 0.1 g, v = 0.001 g^2, lr_t = lr sqrt(0.001) / 0.1 -> step ~ lr * sign(g)
    torch.testing.assert_close(p, torch.tensor([1.0, -2.0], dtype=torch.float64) - 1e-3 * torch.sign(g),
                               rtol=0, atol=1e-7)
