"""Differentiation check at 512x512, batch 4, kernel radius 7 (window 15):
the spatial filter's band gradient and the regression backward, both
computed by the CUDA kernels on the whole batch, against float64.

Spatial filter: central differences (h = 1e-4 relative to |band|) of a
float64 evaluation of the filter at the perturbed pixel (a band value only
changes that pixel's outputs) on 256 random pixels x all 5 band channels;
and the whole gradient against the reference's own gradient kernels, batch
slice by batch slice (the reference op covers slice 0 only).
Tolerances: FD max relative error 2e-3 (floor 1e-3); reference rtol 1e-4
(absolute floor 1e-6 of the gradient's scale).

Regression backward: float64 autograd of oracle/regression_fp64.py on
128x128 crops (origins on the sparsity grid).  A pixel's gradient depends on
data within 4 hw + 2 s + 2 = 38 px, so pixels at least 40 px inside a crop
have their full-image gradient; 256 of them (x 4 inputs x 3 channels) are
compared, and 16 against float64 central differences on the crop (h = 1e-4).
Tolerance, per crop: the image gradients |g - g64| <= 1e-4 max|g64| +
1e-4 |g64|, as the small-image regression-gradient tests (measured: within
1.3e-7 of max|g64|); the albedo and normal gradients 1e-3 max|g64| + 1e-3
|g64|, because each is a sum of per-pair terms w (u r - a beta) that nearly
cancel (the normal equations drive the weighted residuals r to zero), with
u = A^-1 dL/dbeta large where A is ill-conditioned, so the FP32 solve's and
sums' rounding remains in the small result: measured up to 6.6e-4 of
max|g64| at this size (the restatement itself, evaluated in FP32 by torch
autograd, differs from FP64 by 4.2e-4 and 3.2e-4 of max on such a crop).
The finite differences within 5e-4 (their own truncation error).
"""
import numpy as np
import pytest
import torch

from gpu_util import N, T, needs_reference
from helpers import assert_close
from oracle import reference as ref
from oracle import regression_fp64 as r64

pytestmark = pytest.mark.gpu
B, H, W, WIN, SP = 4, 512, 512, 15, 4


def batch_inputs(cd, seed):
    fs = []
    for b in range(B):
        f = cd.synth.make_sequence(H, W, seed=seed + b).frame(2)
        fs.append((np.log1p(f["color"].numpy()), np.log1p(f["color2"].numpy()), f["albedo"].numpy(),
                   f["normal"].numpy()))
    return [np.concatenate([x[i] for x in fs]) for i in range(4)]


def filter_at(imgs, band, win, by, bx, bb):
    """FP64 filter outputs at pixels (bb, by, bx) for band values `band`
    [n, 5]: (acca [n,3], accb [n,3], wsa [n], wsb [n])."""
    ia, ib, al, nr = imgs
    r = win // 2
    off = np.arange(-r, r + 1)
    mir = lambda i, n: np.where(i >= n, 2 * n - 2 - i, np.abs(i))
    yy = mir(by[:, None] + off[None, :], H)                # [n, win]
    xx = mir(bx[:, None] + off[None, :], W)
    g = lambda img: img[bb[:, None, None], yy[:, :, None], xx[:, None, :]]   # [n, win, win, C]
    c = lambda img: img[bb, by, bx][:, None, None, :]
    d = off / r
    pd = d[:, None] ** 2 + d[None, :] ** 2
    dist = lambda img: ((c(img) - g(img)) ** 2).sum(-1)
    dA, dB, dAl, dN = dist(ia), dist(ib), dist(al), dist(nr)
    b_ = band[:, None, None, :]
    wA = np.exp(-b_[..., 0] * dA - b_[..., 2] * dAl - b_[..., 3] * dN - b_[..., 4] * pd)
    wB = np.exp(-b_[..., 1] * dB - b_[..., 2] * dAl - b_[..., 3] * dN - b_[..., 4] * pd)
    return ((wA[..., None] * g(ia)).sum((1, 2)), (wB[..., None] * g(ib)).sum((1, 2)), wA.sum((1, 2)),
            wB.sum((1, 2)))


def test_spatial_filter_gradient_512(cd, cuda):
    ia, ib, al, nr = batch_inputs(cd, seed=31)
    g = torch.Generator(device="cuda:0").manual_seed(32)
    band = torch.clamp(cd.synth.random_band((B, H, W), g, device="cuda:0"), 0.0, 20.0)
    rng = np.random.default_rng(33)
    gs = [rng.standard_normal((B, H, W, c)).astype(np.float32) for c in (3, 3, 1, 1)]
    x = [T(a) for a in (ia, ib, al, nr)] + [band]
    gb = N(cd.ops.spatial_filter_grad(*[T(a) for a in gs], *x, win_size=WIN))
    torch.cuda.synchronize()
    n = 256
    bb, by, bx = rng.integers(B, size=n), rng.integers(H, size=n), rng.integers(W, size=n)
    imgs = [a.astype(np.float64) for a in (ia, ib, al, nr)]
    b64 = N(band).astype(np.float64)[bb, by, bx]            # [n, 5]
    G = [a.astype(np.float64)[bb, by, bx] for a in gs]
    errs = []
    for ch in range(5):
        h = 1e-4 * np.maximum(1.0, np.abs(b64[:, ch]))
        bp, bm = b64.copy(), b64.copy()
        bp[:, ch] += h
        bm[:, ch] -= h
        op, om = filter_at(imgs, bp, WIN, by, bx, bb), filter_at(imgs, bm, WIN, by, bx, bb)
        fd = sum(((a - c) * gg.reshape(a.shape)).reshape(n, -1).sum(1) for a, c, gg in zip(op, om, G)) / (2 * h)
        got = gb[bb, by, bx, ch]
        errs.append(np.abs(got - fd) / np.maximum(np.abs(fd), 1e-3))
    errs = np.concatenate(errs)
    assert errs.max() < 2e-3, f"max relative error {errs.max():.3g} over {errs.size} (pixel, channel) pairs"


@needs_reference
def test_spatial_filter_gradient_512_vs_reference(cd, cuda):
    ia, ib, al, nr = batch_inputs(cd, seed=41)
    g = torch.Generator(device="cuda:0").manual_seed(42)
    band = cd.synth.random_band((B, H, W), g, device="cuda:0")
    rng = np.random.default_rng(43)
    gs = [T(rng.standard_normal((B, H, W, c)).astype(np.float32)) for c in (3, 3, 1, 1)]
    x = [T(a) for a in (ia, ib, al, nr)] + [band]
    gb = N(cd.ops.spatial_filter_grad(*gs, *x, win_size=WIN))
    for b in range(B):
        sl = lambda t: t[b:b + 1].contiguous()
        ref.spatial_filter(*[sl(t) for t in x], WIN)       # the reference's grad reads the forward's partials
        rg = N(ref.spatial_filter_grad(*[sl(t) for t in gs], *[sl(t) for t in x], WIN))
        torch.cuda.synchronize()
        assert_close(gb[b:b + 1], rg, f"band gradient slice {b} vs reference", atol=1e-6 * np.abs(rg).max())


def test_regression_gradient_512(cd, cuda):
    ins = batch_inputs(cd, seed=51)
    rng = np.random.default_rng(52)
    ups = [rng.standard_normal((B, H, W, 3)).astype(np.float32) for _ in range(2)] + \
          [rng.standard_normal((B, H, W, 1)).astype(np.float32) for _ in range(2)]
    got = [N(t) for t in cd.ops.cross_regression_grad(*[T(u) for u in ups], *[T(a) for a in ins], WIN, SP, 1)]
    torch.cuda.synchronize()
    C, margin = 128, 40
    checked, fd_checked = 0, 0
    for k in range(8):
        b = k % B
        oy = int(rng.integers(0, (H - C) // SP + 1)) * SP
        ox = int(rng.integers(0, (W - C) // SP + 1)) * SP
        crop = lambda a: torch.from_numpy(np.ascontiguousarray(a[b:b + 1, oy:oy + C, ox:ox + C])).double()
        x = [crop(a).requires_grad_(True) for a in ins]
        gu = [crop(u) for u in ups]

        def loss(xs):
            return sum((o * g).sum() for o, g in zip(r64.cross_regression(*xs, WIN, SP, 1), gu))

        loss(x).backward()
        g64 = [t.grad.numpy()[0] for t in x]
        qy = rng.integers(margin, C - margin, size=32)
        qx = rng.integers(margin, C - margin, size=32)
        for i in range(4):
            want = g64[i][qy, qx]
            have = got[i][b, oy + qy, ox + qx]
            scale = np.abs(g64[i][margin:C - margin, margin:C - margin]).max()
            tol = 1e-4 if i < 2 else 1e-3   # images | albedo, normal
            bad = np.abs(have - want) > tol * scale + tol * np.abs(want)
            assert not bad.any(), (f"crop {k} input {i}: {bad.sum()} of {bad.size} beyond tolerance, "
                                   f"max err {np.abs(have - want).max():.3g}, scale {scale:.3g}")
        checked += 32
        # two of its pixels against float64 central differences on the crop
        for j in range(2):
            i, c = int(rng.integers(4)), int(rng.integers(3))
            h = 1e-4
            xp = [t.detach().clone() for t in x]
            xm = [t.detach().clone() for t in x]
            xp[i][0, qy[j], qx[j], c] += h
            xm[i][0, qy[j], qx[j], c] -= h
            with torch.no_grad():
                fd = (loss(xp) - loss(xm)).item() / (2 * h)
            have = got[i][b, oy + qy[j], ox + qx[j], c]
            assert abs(have - fd) <= 5e-4 * max(abs(fd), 1.0), (k, i, c, have, fd)
            fd_checked += 1
    assert checked == 256 and fd_checked == 16
