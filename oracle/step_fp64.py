"""Float64 restatement of the whole per-frame train_step, for the precision
report.

TEST INFRASTRUCTURE ONLY.  Follows scripts/main.py:250-313 with:
  log1p                       scripts/main.py:207-212
  cross_regression            oracle/regression_fp64.py (ops/regression.cu.cc:244-500)
  Reproject, 3x3 erosion,     the single-precision C oracle (oracle/oracle.py):
  temporal screening          their outputs are decisions and data moves, and
                              the decisions are the ones under test elsewhere
                              (bit-exact); they are run on the FP64 step's own
                              float32-rounded regression outputs and history
  kernel-predicting U-Net     oracle/unet_torch.py in float64
  spatial filter              filter_fp64 below (ops/regression.cu.cc:84-195)
  aggregation loss            aggregation_fp64 below (scripts/main.py:214-248)
  dL/dparams, Adam            torch.autograd in float64, Keras Adam
Dense over windows and (pixel, centre) pairs: small frames only.
"""
from __future__ import annotations

import numpy as np
import torch

from . import oracle as orc
from . import regression_fp64 as r64
from . import unet_torch as ut


def filter_fp64(imga, imgb, alb, nrm, band, win):
    """Spatial filter forward, [B,H,W,C] tensors (ops/regression.cu.cc:84-195)."""
    B, H, W, _ = imga.shape
    r = win // 2
    idx_y = torch.arange(H).view(H, 1) + torch.arange(-r, r + 1).view(1, -1)
    idx_x = torch.arange(W).view(W, 1) + torch.arange(-r, r + 1).view(1, -1)
    mir = lambda i, n: torch.where(i >= n, 2 * n - 2 - i, i.abs())
    iy, ix = mir(idx_y, H), mir(idx_x, W)

    def win_of(img):  # [B,H,W,C] -> [B,H,W,win,win,C]
        return img[:, iy][:, :, :, ix].permute(0, 1, 3, 2, 4, 5)

    d = torch.arange(-r, r + 1, dtype=imga.dtype) / r
    pd = d.view(-1, 1) ** 2 + d.view(1, -1) ** 2
    dist = lambda img: ((img[:, :, :, None, None, :] - win_of(img)) ** 2).sum(-1)
    dA, dB, dAl, dN = dist(imga), dist(imgb), dist(alb), dist(nrm)
    b = band[:, :, :, None, None, :]
    eA = -b[..., 0] * dA - b[..., 2] * dAl - b[..., 3] * dN - b[..., 4] * pd
    eB = -b[..., 1] * dB - b[..., 2] * dAl - b[..., 3] * dN - b[..., 4] * pd
    wA, wB = eA.exp(), eB.exp()
    acca = (wA[..., None] * win_of(imga)).sum((3, 4))
    accb = (wB[..., None] * win_of(imgb)).sum((3, 4))
    return acca, accb, wA.sum((3, 4))[..., None], wB.sum((3, 4))[..., None]


def aggregation_fp64(sum1, sumw1, sum2, sumw2, alpha, success, success_prev, prev_out, opacity, label1, label2,
                     prev_label1, prev_label2):
    """aggregation_loss (scripts/main.py:214-248), differentiable.
    Returns (out_log, out, loss, avg_loss)."""
    out1 = sum1 / (sumw1 + 1e-4)
    out2 = sum2 / (sumw2 + 1e-4)
    out = (sum1 + sum2) / (sumw1 + sumw2 + 1e-4)
    op = torch.where(opacity > 0, 1.0, 0.0).to(out.dtype)
    s = success * success_prev
    a = s * alpha + (1 - s)
    out = (a * out + (1 - a) * prev_out) * op
    o1 = a * out1 + (1 - a) * prev_out
    o2 = a * out2 + (1 - a) * prev_out
    spatial = ((o1 - label1) ** 2 / (label1 ** 2 + 1e-2) + (o2 - label2) ** 2 / (label2 ** 2 + 1e-2)) * 0.5
    temporal = ((o1 - prev_label1) ** 2 / (prev_label1 ** 2 + 1e-2)
                + (o2 - prev_label2) ** 2 / (prev_label2 ** 2 + 1e-2)) * 0.5
    loss = (spatial + temporal) * 0.5 * op
    return out, torch.clamp(torch.expm1(out), min=0.0), loss, loss.mean()


class StepFP64:
    """One stream's train_step in float64 with its own history and Adam state."""

    def __init__(self, params: np.ndarray, regression_width=15, filter_width=11, sparsity=4, lr=1e-3):
        self.p = torch.from_numpy(np.asarray(params, np.float64)).clone()
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step = 0
        self.lr = lr
        self.rw, self.fw, self.sp = regression_width, filter_width, sparsity
        self.hist = None

    def __call__(self, f):
        """f: dict of [1,H,W,C] float32 numpy arrays; returns float64 numpy outputs."""
        T = lambda a: torch.from_numpy(np.asarray(a, np.float64))
        _, H, W, _ = f["color"].shape
        if self.hist is None:
            z = np.zeros((1, H, W, 3), np.float32)
            self.hist = dict(out_log=z, ols1=z, ols2=z, linz=z, nrm=z)
        h = self.hist
        y1, y2 = torch.log1p(T(f["color"])), torch.log1p(T(f["color2"]))
        alb, nrm = T(f["albedo"]), T(f["normal"])
        ols1, ols2, _, _ = r64.cross_regression(y1, y2, alb, nrm, self.rw, self.sp, 1)
        o1f, o2f = ols1.numpy().astype(np.float32), ols2.numpy().astype(np.float32)
        one = np.ones((1, H, W, 1), np.float32)
        succ, rep = orc.reproject(f["mvec"], [h["out_log"], h["ols1"], h["ols2"]], f["linearZ"], h["linz"],
                                  f["normal"], h["nrm"], f["pnFwidth"], one, one)
        ero = orc.erode3x3(succ)
        po, p1, p2, sp = orc.temporal_screening(o1f, o2f, rep[0], rep[1], rep[2], ero, 7, 1)
        po, p1, p2, sp, ero = T(po), T(p1), T(p2), T(sp), T(ero)
        params = self.p.clone().requires_grad_(True)
        band, alpha = ut.forward(params, ols1, ols2, po, alb, nrm)
        band.retain_grad()
        alpha.retain_grad()
        s1, s2, w1, w2 = filter_fp64(ols1, ols2, alb, nrm, band, self.fw)
        out_log, out, loss, avg = aggregation_fp64(s1, w1, s2, w2, alpha, ero, sp, po, T(f["opacity"]), ols2, ols1,
                                                   p2, p1)
        avg.backward()
        self.step += 1
        ut.adam_keras(self.p, params.grad.detach(), self.m, self.v, self.step, lr=self.lr)
        self.hist = dict(out_log=out_log.detach().numpy().astype(np.float32), ols1=o1f, ols2=o2f,
                         linz=f["linearZ"], nrm=f["normal"])
        d = lambda t: t.detach().numpy()
        return {"ols1": d(ols1), "ols2": d(ols2), "band": d(band), "alpha": d(alpha), "out_log": d(out_log),
                "out": d(out), "avg_loss": float(avg), "g_band": d(band.grad), "g_alpha": d(alpha.grad),
                "params": self.p.numpy().copy()}
