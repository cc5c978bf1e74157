"""PyTorch restatement of the reference's kernel-predicting U-Net, for tests.

TEST INFRASTRUCTURE ONLY: the checker of the tensor-core U-Net kernels,
never a product path.  Keras semantics of scripts/main.py:83-118
(TensorFlow 2.16.1 is not installed here, so parity with Keras itself is
unpinned; this follows the layers' documented definitions):

  Conv2D(k=3, 'same')           cross-correlation, zero padding, kernel
                                [kh][kw][cin][cout], bias, ReLU (:84-98)
  MaxPooling2D(2)               2x2, stride 2, 'valid' (:86, :89)
  Conv2DTranspose(k=1, s=2)     out[2i, 2j] = K x[i, j] + b, other positions
                                b; kernel [1][1][cout][cin] (:92, :96)
  Concatenate(axis=-1)          [c3_3, c2_2], [c4_3, c1_2] (:93, :97)
  head Conv2D(6, 1), float32    band = 1 / (p^2 + 1e-4), alpha = sigmoid
                                (:106-111)

``bf16=True`` rounds what the GPU path stores in bf16 (the packed input,
every activation, the 3x3 kernels) so the comparison isolates accumulation
order; ``bf16=False`` in float64 is the precision oracle.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F

SHAPES_LAYERS = [("conv", 15, 8), ("conv", 8, 8), ("conv", 8, 16), ("conv", 16, 16), ("conv", 16, 32),
                 ("conv", 32, 32), ("tconv", 32, 32), ("conv", 48, 16), ("conv", 16, 16), ("tconv", 16, 16),
                 ("conv", 24, 8), ("head", 8, 6)]


def unflatten(flat: torch.Tensor):
    out, o = [], 0
    for kind, cin, cout in SHAPES_LAYERS:
        ks = (3, 3, cin, cout) if kind == "conv" else ((1, 1, cout, cin) if kind == "tconv" else (1, 1, cin, cout))
        n = 1
        for d in ks:
            n *= d
        out.append((kind, flat[o:o + n].reshape(ks), flat[o + n:o + n + cout]))
        o += n + cout
    return out


def _rb(x, on):
    return x.to(torch.bfloat16).to(x.dtype) if on else x


def conv3x3(x, K, b, relu=True):
    """x NCHW; K [3,3,cin,cout] Keras layout."""
    w = K.permute(3, 2, 0, 1)   # [cout, cin, kh, kw]
    y = F.conv2d(x, w, b, padding=1)
    return F.relu(y) if relu else y


def tconv(x, K, b):
    """Conv2DTranspose(kernel 1, stride 2, 'same'): K [1,1,cout,cin]."""
    Bn, C, H, W = x.shape
    w = K[0, 0]                                   # [cout, cin]
    y = torch.einsum("oc,bchw->bohw", w, x)
    out = b.view(1, -1, 1, 1).expand(Bn, w.shape[0], 2 * H, 2 * W).clone()
    out[:, :, 0::2, 0::2] = out[:, :, 0::2, 0::2] + y
    return out


def forward(params: torch.Tensor, ols1, ols2, prev_out, albedo, normal, bf16: bool = False, keep=None):
    """Inputs NHWC [B,H,W,3]; returns (band [B,H,W,5], alpha [B,H,W,1]).
    If `keep` is a dict, the NCHW activations are stored in it by name."""
    L = unflatten(params)
    rb = lambda t: _rb(t, bf16)
    kw = lambda i: rb(L[i][1])
    x = torch.cat([ols1, ols2, prev_out, albedo, normal], -1).permute(0, 3, 1, 2)
    x = rb(x)
    c11 = rb(conv3x3(x, kw(0), L[0][2]))
    c12 = rb(conv3x3(c11, kw(1), L[1][2]))
    c13 = F.max_pool2d(c12, 2)
    c21 = rb(conv3x3(c13, kw(2), L[2][2]))
    c22 = rb(conv3x3(c21, kw(3), L[3][2]))
    c23 = F.max_pool2d(c22, 2)
    c31 = rb(conv3x3(c23, kw(4), L[4][2]))
    c32 = rb(conv3x3(c31, kw(5), L[5][2]))
    c33 = rb(tconv(c32, L[6][1], L[6][2]))
    c41 = rb(conv3x3(torch.cat([c33, c22], 1), kw(7), L[7][2]))
    c42 = rb(conv3x3(c41, kw(8), L[8][2]))
    c43 = rb(tconv(c42, L[9][1], L[9][2]))
    c51 = rb(conv3x3(torch.cat([c43, c12], 1), kw(10), L[10][2]))
    Kh, bh = L[11][1][0, 0], L[11][2]            # [8, 6]
    p = torch.einsum("bchw,co->bhwo", c51, Kh) + bh
    band = 1.0 / (p[..., :5] ** 2 + 1e-4)
    alpha = torch.sigmoid(p[..., 5:])
    if keep is not None:
        keep.update(x=x, c11=c11, c12=c12, c13=c13, c21=c21, c22=c22, c23=c23, c31=c31, c32=c32, c33=c33,
                    c41=c41, c42=c42, c43=c43, c51=c51)
    return band, alpha


def adam_keras(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-7):
    """One keras.optimizers.Adam update (in place), step >= 1."""
    m += (g - m) * (1 - b1)
    v += (g * g - v) * (1 - b2)
    lr_t = lr * (1 - b2 ** step) ** 0.5 / (1 - b1 ** step)
    p -= (m * lr_t) / (v.sqrt() + eps)
    return p, m, v
