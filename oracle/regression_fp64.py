"""Differentiable FP64 restatement of CrossRegression, for gradient checks.

TEST INFRASTRUCTURE ONLY.  The reference registers no gradient for
CrossRegression (scripts/ops.py:23-32), so the backward kernels of this
repository are checked against torch.autograd through this float64
restatement of the forward (and this restatement against central finite
differences).  It follows the same formulas as oracle/cd_oracle.c:

  variance      ops/regression.cu.cc:244-276  (in-bounds 3x3 mean without the centre)
  regression    ops/regression.cu.cc:367-475  (reflect-101 window, ridge 1e-3)
  block recon   ops/regression.cu.cc:289-365  (centre range with the iDivUp rule)

The reconstruction gathers, per output pixel, the centres of its clamped
range (at most ceil((2 hw + 1) / s) + 1 per axis); small and medium images.
The Cholesky pivot clamp max(1e-5, .) of the reference never binds for the
ridge-regularised systems (their Schur complements are >= 1e-3) and is left
out; the solve is torch.linalg.solve.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F


def _mirror(i: torch.Tensor, n: int) -> torch.Tensor:
    return torch.where(i >= n, 2 * n - 2 - i, i.abs())


def idivup_c(a: int, b: int) -> int:
    """iDivUp with C's truncating division and remainder."""
    q = abs(a) // abs(b)
    q = q if (a >= 0) == (b >= 0) else -q
    r = a - b * q
    return q + 1 if r != 0 else q


def variance(img: torch.Tensor) -> torch.Tensor:
    """[B,H,W,3] -> [B,H,W,1]."""
    x = img.permute(0, 3, 1, 2)
    ones = torch.ones_like(x[:, :1])
    k = torch.ones((1, 1, 3, 3), dtype=img.dtype, device=img.device)
    s = F.conv2d(F.pad(x, (1, 1, 1, 1)), k.expand(3, 1, 3, 3), groups=3) - x
    n = F.conv2d(F.pad(ones, (1, 1, 1, 1)), k) - 1
    mean = s / n
    return ((mean - x) ** 2).sum(1, keepdim=True).permute(0, 2, 3, 1)


def _branch(y, f, v, alb, nrm, win, sp, rs):
    B, H, W, _ = f.shape
    hw = win // 2
    Hs, Ws = H // sp, W // sp
    dev = f.device
    s = torch.sqrt(v)
    cy = torch.arange(Hs, device=dev) * sp
    cx = torch.arange(Ws, device=dev) * sp
    off = torch.arange(-hw, hw + 1, device=dev)
    ty = _mirror(cy[:, None] + off[None, :], H)            # [Hs, win]
    tx = _mirror(cx[:, None] + off[None, :], W)            # [Ws, win]

    def taps(img):   # [B,H,W,C] -> [B,Hs,Ws,win*win,C]
        g = img[:, ty][:, :, :, tx]                        # [B,Hs,win,Ws,win,C]
        return g.permute(0, 1, 3, 2, 4, 5).reshape(B, Hs, Ws, win * win, img.shape[-1])

    def centres(img):
        return img[:, cy][:, :, cx][:, :, :, None]          # [B,Hs,Ws,1,C]

    ft, yt, at, nt, vt, st = taps(f), taps(y), taps(alb), taps(nrm), taps(v), taps(s)
    fc, ac, nc, vc, sc = centres(f), centres(alb), centres(nrm), centres(v), centres(s)
    den = sc + st + 1e-2                                    # [..,T,1]
    df = ft - fc
    d1 = df / den                                           # [..,T,3]
    da = at - ac
    dn = nt - nc
    dist = (df ** 2).sum(-1, keepdim=True) / (vc + vt + 1e-4)
    w = torch.exp(-dist) + 1e-7                             # [..,T,1]
    ones = torch.ones_like(d1)
    X = torch.stack([ones, d1, da, dn[..., 0:1].expand_as(d1), dn[..., 1:2].expand_as(d1),
                     dn[..., 2:3].expand_as(d1)], -1)      # [B,Hs,Ws,T,3,6]
    A = torch.einsum("bhwtki,bhwt,bhwtkj->bhwkij", X, w[..., 0], X)
    A = A + 1e-3 * torch.eye(6, dtype=f.dtype, device=dev)
    b = torch.einsum("bhwtki,bhwt,bhwtk->bhwki", X, w[..., 0], yt)
    beta = torch.linalg.solve(A, b.unsqueeze(-1)).squeeze(-1)   # [B,Hs,Ws,3,6]

    # block reconstruction: for every output pixel, the centres of its clamped
    # iDivUp range along each axis (at most K per axis), gathered with a mask
    Hr, Wr = H // rs, W // rs

    def ranges(n_out, n, ncen):
        lo = [max(0, idivup_c(p * rs - hw, sp)) for p in range(n_out)]
        hi = [min((n - 1) // sp, (p * rs + hw) // sp) for p in range(n_out)]
        K = max(h - l + 1 for l, h in zip(lo, hi))
        idx = torch.tensor([[min(l + k, ncen - 1) for k in range(K)] for l in lo], device=dev)
        ok = torch.tensor([[l + k <= h for k in range(K)] for l, h in zip(lo, hi)], device=dev)
        return idx, ok                                       # [n_out, K]

    jy, oky = ranges(Hr, H, Hs)
    ix, okx = ranges(Wr, W, Ws)
    Ky, Kx = jy.shape[1], ix.shape[1]
    py = torch.arange(Hr, device=dev) * rs
    px = torch.arange(Wr, device=dev) * rs

    def at_out(img):                                        # [B,Hr,Wr,1,1,C]
        return img[:, py][:, :, px][:, :, :, None, None, :]

    def at_cen(img):                                        # [B,Hr,Wr,Ky,Kx,C]
        g = img[:, cy][:, :, cx]                            # [B,Hs,Ws,C]
        return g[:, jy][:, :, :, ix].permute(0, 1, 3, 2, 4, 5)

    fp, ap, np_, vp, sp_ = at_out(f), at_out(alb), at_out(nrm), at_out(v), at_out(s)
    fcc, acc, ncc, vcc, scc = at_cen(f), at_cen(alb), at_cen(nrm), at_cen(v), at_cen(s)
    den2 = sp_ + scc + 1e-2
    dfp = fp - fcc
    d1p = dfp / den2
    dap = ap - acc
    dnp = np_ - ncc
    Bc = beta[:, jy][:, :, :, ix].permute(0, 1, 3, 2, 4, 5, 6)   # [B,Hr,Wr,Ky,Kx,3,6]
    pred = (Bc[..., 0] + Bc[..., 1] * d1p + Bc[..., 2] * dap + Bc[..., 3] * dnp[..., 0:1]
            + Bc[..., 4] * dnp[..., 1:2] + Bc[..., 5] * dnp[..., 2:3])
    distp = (dfp ** 2).sum(-1, keepdim=True) / (vp + vcc + 1e-4)
    mask = (oky[:, None, :, None] & okx[None, :, None, :]).to(f.dtype)[None, ..., None]   # [1,Hr,Wr,Ky,Kx,1]
    wp = (torch.exp(-distp) + 1e-7) * mask
    num = (wp * pred).sum((3, 4))
    den_sum = wp.sum((3, 4))
    return torch.relu(num / torch.clamp(den_sum, min=1e-7))


def cross_regression(imga, imgb, albedo, normal, win_size, sparsity, recon_scale=1):
    """(outa, outb, vara, varb) in the dtype of the inputs (float64 for checks)."""
    va, vb = variance(imga), variance(imgb)
    outa = _branch(imgb, imga, va, albedo, normal, win_size, sparsity, recon_scale)
    outb = _branch(imga, imgb, vb, albedo, normal, win_size, sparsity, recon_scale)
    return outa, outb, va, vb
