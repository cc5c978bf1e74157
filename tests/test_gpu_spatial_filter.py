"""SpatialFilter forward and band gradient on the GPU: against the oracle,
the golden reference outputs and the live reference kernels (rtol 1e-4),
through autograd, and the gradient against FP64 central finite differences."""
import numpy as np
import pytest
import torch

from gpu_util import N, T, frames, needs_reference
from helpers import assert_close, golden, golden_names
from oracle import oracle as orc
from oracle import reference as ref

from oracle.step_fp64 import filter_fp64  # noqa: E402

pytestmark = pytest.mark.gpu


def inputs(cd, H, W, seed, B=1):
    fs = [frames(cd, H, W, seed=seed + b)[1] for b in range(B)]
    cat = lambda k: np.concatenate([f[k] for f in fs])
    g = torch.Generator().manual_seed(seed)
    band = cd.synth.random_band((B, H, W), g).numpy()
    return np.log1p(cat("color")), np.log1p(cat("color2")), cat("albedo"), cat("normal"), band


def upstream(B, H, W, seed):
    rng = np.random.default_rng(seed)
    return [rng.normal(size=(B, H, W, c)).astype(np.float32) for c in (3, 3, 1, 1)]


@pytest.mark.parametrize("name", golden_names("spatial_filter_"))
def test_golden(cd, cuda, name):
    g = golden(name)
    win = int(g["attr_win_size"])
    ins = [T(g[k]) for k in ("in_imga", "in_imgb", "in_albedo", "in_normal", "in_band")]
    o = cd.ops.spatial_filter(*ins, win_size=win)
    gs = [T(g[k]) for k in ("in_grad_acca", "in_grad_accb", "in_grad_wgtsuma", "in_grad_wgtsumb")]
    gb = cd.ops.spatial_filter_grad(*gs, *ins, win_size=win)
    torch.cuda.synchronize()
    for x, key in zip(o, ("ref_acca", "ref_accb", "ref_wgtsuma", "ref_wgtsumb")):
        assert_close(N(x), g[key], f"{name} {key}", atol=1e-5)
    scale = np.abs(g["ref_grad_band"]).max()
    assert_close(N(gb), g["ref_grad_band"], f"{name} grad_band", atol=1e-6 * scale)


@pytest.mark.parametrize("H,W,B,win", [(128, 160, 2, 11), (96, 96, 1, 7), (70, 90, 1, 15), (33, 47, 1, 3),
                                       (64, 64, 1, 21)])
def test_vs_oracle(cd, cuda, H, W, B, win):
    x = inputs(cd, H, W, seed=win, B=B)
    gs = upstream(B, H, W, seed=win)
    o = cd.ops.spatial_filter(*[T(a) for a in x], win_size=win)
    gb = cd.ops.spatial_filter_grad(*[T(a) for a in gs], *[T(a) for a in x], win_size=win)
    torch.cuda.synchronize()
    r = orc.spatial_filter(*x, win, partials=True)
    rg = orc.spatial_filter_grad_from_partials(*gs, r[4], r[5])
    for i, nm in enumerate(("acca", "accb", "wsa", "wsb")):
        assert_close(N(o[i]), r[i], nm, atol=1e-5)
    assert_close(N(gb), rg, "grad_band", atol=1e-6 * np.abs(rg).max())


@needs_reference
def test_vs_reference_kernels(cd, cuda):
    x = [T(a) for a in inputs(cd, 256, 320, seed=4)]
    gs = [T(a) for a in upstream(1, 256, 320, seed=4)]
    o = cd.ops.spatial_filter(*x, win_size=11)
    gb = cd.ops.spatial_filter_grad(*gs, *x, win_size=11)
    r = ref.spatial_filter(*x, 11)
    rg = ref.spatial_filter_grad(*gs, *x, 11)
    torch.cuda.synchronize()
    for i in range(4):
        assert_close(N(o[i]), N(r[i]), f"out{i} vs reference", atol=1e-5)
    assert_close(N(gb), N(rg), "grad vs reference", atol=1e-6 * N(rg).__abs__().max())


def test_autograd_matches_grad_op(cd, cuda):
    x = [T(a) for a in inputs(cd, 48, 64, seed=8)]
    band = x[4].clone().requires_grad_(True)
    gs = [T(a) for a in upstream(1, 48, 64, seed=9)]
    o = cd.ops.spatial_filter(x[0], x[1], x[2], x[3], band, win_size=9)
    loss = sum((oi * gi).sum() for oi, gi in zip(o, gs))
    loss.backward()
    direct = cd.ops.spatial_filter_grad(*gs, *x, win_size=9)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(N(band.grad), N(direct))


def test_gradient_vs_fp64_finite_differences(cd, cuda):
    """Central differences (h = 1e-4, relative to |band|) of the FP64
    restatement against the FP32 kernel's analytic gradient on 256 random
    (pixel, band channel) pairs."""
    B, H, W, win = 2, 24, 28, 15
    x = inputs(cd, H, W, seed=12, B=B)
    x = list(x)
    x[4] = np.clip(x[4], 0.0, 20.0).astype(np.float32)    # keep exp() in a well-scaled range
    gs = upstream(B, H, W, seed=13)
    gb = N(cd.ops.spatial_filter_grad(*[T(a) for a in gs], *[T(a) for a in x], win_size=win))
    xd = [torch.from_numpy(a).double() for a in x]
    gd = [torch.from_numpy(a).double() for a in gs]
    loss = lambda band: sum((o * g).sum() for o, g in zip(filter_fp64(*xd[:4], band, win), gd)).item()
    rng = np.random.default_rng(14)
    errs = []
    for _ in range(256):
        b, yy, xx, ch = rng.integers(B), rng.integers(H), rng.integers(W), rng.integers(5)
        h = 1e-4 * max(1.0, abs(float(x[4][b, yy, xx, ch])))
        bp, bm = xd[4].clone(), xd[4].clone()
        bp[b, yy, xx, ch] += h
        bm[b, yy, xx, ch] -= h
        fd = (loss(bp) - loss(bm)) / (2 * h)
        errs.append(abs(gb[b, yy, xx, ch] - fd) / max(abs(fd), 1e-3))
    assert np.max(errs) < 2e-3, f"max relative error {np.max(errs):.3g}"


def test_image_gradients_are_none(cd, cuda):
    x = [T(a).requires_grad_(True) for a in inputs(cd, 16, 16, seed=1)]
    o = cd.ops.spatial_filter(*x, win_size=5)
    o[0].sum().backward()
    assert x[0].grad is None and x[3].grad is None and x[4].grad is not None


def test_argument_errors(cd, cuda):
    x = torch.zeros((1, 8, 8, 3), device=cuda)
    b = torch.zeros((1, 8, 8, 5), device=cuda)
    with pytest.raises(ValueError):
        cd.ops.spatial_filter(x, x, x, x, b, win_size=0)
    with pytest.raises(ValueError):
        cd.ops.spatial_filter(x, x, x, x, b, win_size=17)          # radius 8 >= H
    with pytest.raises(ValueError):
        cd.ops.spatial_filter(x, x, x, x, b[..., :4], win_size=3)


def test_stored_partials_variant_is_identical(cd, cuda):
    """The stored-partials design (the reference's) gives the recomputing
    kernels' results bit for bit."""
    x = [T(a) for a in inputs(cd, 40, 72, seed=21, B=2)]
    gs = [T(a) for a in upstream(2, 40, 72, seed=22)]
    for win in (7, 15):
        o = cd.ops.spatial_filter(*x, win_size=win)
        gb = cd.ops.spatial_filter_grad(*gs, *x, win_size=win)
        o2 = cd.ops.spatial_filter_stored(*x, win_size=win)
        gb2 = cd.ops.spatial_filter_grad_stored(*gs, o2[4])
        torch.cuda.synchronize()
        for a, b in zip(o, o2[:4]):
            np.testing.assert_array_equal(N(a), N(b))
        np.testing.assert_array_equal(N(gb), N(gb2))
