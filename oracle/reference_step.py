"""The reference's per-frame step (scripts/main.py:250-313) chained on the
reference's own CUDA kernels (oracle/reference.py), with the reference's
XLA parts restated in eager PyTorch FP32 (log1p, the aggregation loss and
its gradient).

TEST INFRASTRUCTURE ONLY: the reference side of the chained-sequence parity
tests and the reference arm of bench.py.  Tensors are torch CUDA tensors,
NHWC float32.

Step order and attributes (scripts/main.py:250-313; history hand-off
:323-341, zero history before the first frame :323-330):
  y = log1p(colour);  ols1, ols2 = CrossRegression(y1, y2, albedo, normal)
  success, [prev out_log, ols1, ols2] = Reproject(...) with all-ones opacity
  eroded = erosion2d(float(success)) (3x3, in-bounds min)
  prev_out, prev_ols1, prev_ols2, success_prev = TemporalScreening(7, 1)
  sums = SpatialFilter(ols1, ols2, albedo, normal, band, 11)
  aggregation loss with the labels crossed (label1 = ols2, label2 = ols1)
  g_band = SpatialFilterGrad(...)
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from . import reference as ref


@dataclass
class RefHistory:
    """What the reference carries from one frame to the next."""
    out_log: torch.Tensor
    ols1: torch.Tensor
    ols2: torch.Tensor
    linearZ: torch.Tensor
    normal: torch.Tensor

    @staticmethod
    def zeros(B, H, W, device) -> "RefHistory":
        z = lambda: torch.zeros((B, H, W, 3), dtype=torch.float32, device=device)
        return RefHistory(z(), z(), z(), z(), z())

    def clone(self) -> "RefHistory":
        return RefHistory(*(t.clone() for t in (self.out_log, self.ols1, self.ols2, self.linearZ, self.normal)))


def aggregation_forward_backward(sum1, sumw1, sum2, sumw2, alpha, success, success_prev, prev_out,
                                 opacity, label1, label2, prev_label1, prev_label2):
    """Eager PyTorch restatement of aggregation_loss (scripts/main.py:214-248,
    an XLA function in the reference, not one of its CUDA ops) and its
    gradient with respect to (sum1, sumw1, sum2, sumw2, alpha) in closed form
    (the gradient TF's tape takes through it, :289-302): the FP32 reference
    the CUDA aggregation kernels are tested against, and the glue between the
    reference's kernels in ReferenceStep.

    Returns (out, out_linear, loss, avg_loss, g_sum1, g_sumw1, g_sum2, g_sumw2, g_alpha).
    """
    e = 1e-4
    d1 = sumw1 + e
    d2 = sumw2 + e
    o1s = sum1 / d1
    o2s = sum2 / d2
    out = (sum1 + sum2) / (sumw1 + sumw2 + e)
    op = torch.where(opacity > 0, 1.0, 0.0).to(sum1.dtype)
    s = success * success_prev
    a = s * alpha + (1 - s)
    out = (a * out + (1 - a) * prev_out) * op
    o1 = a * o1s + (1 - a) * prev_out
    o2 = a * o2s + (1 - a) * prev_out
    n1, n2 = label1 * label1 + 1e-2, label2 * label2 + 1e-2
    p1, p2 = prev_label1 * prev_label1 + 1e-2, prev_label2 * prev_label2 + 1e-2
    spatial = ((o1 - label1) ** 2 / n1 + (o2 - label2) ** 2 / n2) * 0.5
    temporal = ((o1 - prev_label1) ** 2 / p1 + (o2 - prev_label2) ** 2 / p2) * 0.5
    loss = (spatial + temporal) * 0.5 * op
    avg = loss.mean()
    c = 0.5 * 0.5 * op / loss.numel()
    g_o1 = c * (2 * (o1 - label1) / n1 + 2 * (o1 - prev_label1) / p1)
    g_o2 = c * (2 * (o2 - label2) / n2 + 2 * (o2 - prev_label2) / p2)
    g_sum1 = g_o1 * a / d1
    g_sum2 = g_o2 * a / d2
    g_sumw1 = -(g_o1 * a * sum1).sum(-1, keepdim=True) / (d1 * d1)
    g_sumw2 = -(g_o2 * a * sum2).sum(-1, keepdim=True) / (d2 * d2)
    g_alpha = (s * (g_o1 * (o1s - prev_out) + g_o2 * (o2s - prev_out))).sum(-1, keepdim=True)
    return (out, torch.clamp(torch.expm1(out), min=0.0), loss, avg,
            g_sum1, g_sumw1, g_sum2, g_sumw2, g_alpha)


class ReferenceStep:
    """One stream's step on the reference's kernels.  Band and alpha are
    given (the network is not part of this chain).  ``step(frame)`` returns
    every intermediate of the frame; ``step.history`` is what the next frame
    reads (None before the first frame: zeros)."""

    def __init__(self, regression_width, sparsity, filter_width, win_curr, win_prev, band, alpha):
        self.win, self.sp, self.fwin = int(regression_width), int(sparsity), int(filter_width)
        self.win_curr, self.win_prev = int(win_curr), int(win_prev)
        self.band, self.alpha = band, alpha
        self.history = None

    def __call__(self, f):
        B, H, W, _ = f["color"].shape
        if self.history is None:
            self.history = RefHistory.zeros(B, H, W, f["color"].device)
        h = self.history
        y1, y2 = torch.log1p(f["color"]), torch.log1p(f["color2"])
        ols1, ols2, _, _ = ref.cross_regression(y1, y2, f["albedo"], f["normal"], self.win, self.sp)
        ones1 = torch.ones((B, H, W, 1), device=y1.device)
        succ, rep = ref.reproject(f["mvec"], [h.out_log, h.ols1, h.ols2], f["linearZ"], h.linearZ, f["normal"],
                                  h.normal, f["pnFwidth"], ones1, ones1)
        ero = ref.erode3x3(succ)
        po, p1, p2, sp = ref.temporal_screening(ols1, ols2, rep[0], rep[1], rep[2], ero, self.win_curr,
                                                self.win_prev)
        s1, s2, w1, w2 = ref.spatial_filter(ols1, ols2, f["albedo"], f["normal"], self.band, self.fwin)
        out_log, out, loss, avg, g1, gw1, g2, gw2, ga = aggregation_forward_backward(
            s1, w1, s2, w2, self.alpha, ero, sp, po, f["opacity"], ols2, ols1, p2, p1)
        gb = ref.spatial_filter_grad(g1, g2, gw1, gw2, ols1, ols2, f["albedo"], f["normal"], self.band,
                                     self.fwin)
        self.history = RefHistory(out_log, ols1, ols2, f["linearZ"], f["normal"])
        return {"y1": y1, "y2": y2, "ols1": ols1, "ols2": ols2, "success": succ, "reprojected": rep,
                "eroded": ero, "prev_out": po, "prev_ols1": p1, "prev_ols2": p2, "success_prev": sp,
                "sum1": s1, "sum2": s2, "sumw1": w1, "sumw2": w2, "out_log": out_log, "out": out,
                "loss": loss, "avg_loss": avg, "g_sum1": g1, "g_sumw1": gw1, "g_sum2": g2, "g_sumw2": gw2,
                "g_alpha": ga, "g_band": gb}
