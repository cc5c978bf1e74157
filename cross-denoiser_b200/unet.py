"""The reference's kernel-predicting U-Net with its online Adam update
(scripts/main.py:74-118 network, :81 optimizer, :289-303 tape and update),
on the tensor-core kernels behind cd_unet_forward / cd_unet_backward /
cd_adam_update.

``UNet`` is a FrameStep predictor: calling it predicts (band, alpha) for a
frame; ``on_gradients(g_band, g_alpha)`` back-propagates dL/dband and
dL/dalpha and applies one Adam step, as the reference's train_step does
once per frame.
"""
from __future__ import annotations

import ctypes
from typing import List, Tuple

import numpy as np
import torch

from . import _lib

LEARNING_RATE = 1e-3        # scripts/main.py:74
BETA1, BETA2, EPSILON = 0.9, 0.999, 1e-7   # keras.optimizers.Adam defaults

# (kind, cin, cout) in the model's trainable-variable order (scripts/main.py:83-108)
LAYERS: List[Tuple[str, int, int]] = [
    ("conv", 15, 8), ("conv", 8, 8), ("conv", 8, 16), ("conv", 16, 16), ("conv", 16, 32), ("conv", 32, 32),
    ("tconv", 32, 32), ("conv", 48, 16), ("conv", 16, 16), ("tconv", 16, 16), ("conv", 24, 8), ("head", 8, 6),
]


def kernel_shape(kind: str, cin: int, cout: int) -> Tuple[int, ...]:
    """Keras kernel shape: Conv2D (kh, kw, cin, cout), Conv2DTranspose (1, 1, cout, cin)."""
    if kind == "conv":
        return (3, 3, cin, cout)
    if kind == "tconv":
        return (1, 1, cout, cin)
    return (1, 1, cin, cout)


def param_shapes() -> List[Tuple[int, ...]]:
    out = []
    for kind, cin, cout in LAYERS:
        out += [kernel_shape(kind, cin, cout), (cout,)]
    return out


def param_count() -> int:
    return int(sum(np.prod(s) for s in param_shapes()))


def glorot_init(seed: int = 1234) -> np.ndarray:
    """Keras defaults: glorot_uniform kernels (limit sqrt(6 / (fan_in +
    fan_out)), fans from the kernel shape's last two axes times the receptive
    field), zero biases.  Seeded with numpy, so not TensorFlow's draw."""
    rng = np.random.default_rng(seed)
    parts = []
    for shape in param_shapes():
        if len(shape) == 1:
            parts.append(np.zeros(shape, np.float32))
            continue
        rf = shape[0] * shape[1]
        fan_in, fan_out = shape[2] * rf, shape[3] * rf
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        parts.append(rng.uniform(-lim, lim, size=shape).astype(np.float32))
    return np.concatenate([p.ravel() for p in parts])


def split_params(flat) -> list:
    """Views of the flat buffer in Keras shapes."""
    out, o = [], 0
    for shape in param_shapes():
        n = int(np.prod(shape))
        out.append(flat[o:o + n].reshape(shape))
        o += n
    return out


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class UNet:
    """Parameters, Adam state and workspace of one stream's network."""

    def __init__(self, device="cuda:0", seed: int = 1234, lr: float = LEARNING_RATE, params=None):
        L = _lib.lib()
        self.n = int(L.cd_unet_param_count())
        assert self.n == param_count() == 31414
        init = glorot_init(seed) if params is None else np.asarray(params, np.float32)
        self.device = torch.device(device)
        self.params = torch.from_numpy(init.copy()).to(self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.lr = float(lr)
        self.step = torch.zeros((1,), dtype=torch.int32, device=self.device)   # optimizer iterations
        self._shape = None
        self.ws = None
        # host copy of the workspace's error flag, refreshed asynchronously
        # after every training update (enqueue_error_readback)
        self.flag_host = torch.zeros((1,), dtype=torch.int32).pin_memory()

    def _workspace(self, B, H, W):
        if self._shape != (B, H, W):
            nbytes = int(_lib.lib().cd_unet_workspace_size(B, H, W))
            if nbytes == 0:
                raise ValueError(f"unet: unsupported frame shape B={B} H={H} W={W} (H, W multiples of 4)")
            self.ws = torch.zeros((nbytes,), dtype=torch.uint8, device=self.device)
            self._shape = (B, H, W)
        return self.ws

    def error_flag(self) -> int:
        """The workspace's error flag, read synchronously: 0 while every bounded
        wait of the tensor-core kernels completed, 1 after a wait for a bulk
        copy ran out, 2 after a wait for an MMA batch ran out.  Never cleared."""
        return int(self.ws[:4].view(torch.int32).item()) if self.ws is not None else 0

    def enqueue_error_readback(self):
        """Copy the error flag to pinned host memory on the current stream
        (no synchronisation); raise_if_failed reads the copy.  Not for use
        inside a CUDA-graph capture."""
        if self.ws is not None:
            self.flag_host.copy_(self.ws[:4].view(torch.int32), non_blocking=True)

    def raise_if_failed(self):
        """Raise UNetTimeoutError if the last flag copy that has landed is
        nonzero.  Reads host memory only: an error is seen once the copy
        enqueued after the failing frame has completed.  After an error the
        network's outputs and parameters are invalid and later kernels of
        the process are suspect (a timed-out CTA may have left copies or MMAs
        writing its shared memory or TMEM)."""
        f = int(self.flag_host[0])
        if f:
            what = "a bulk copy into shared memory" if f == 1 else "an MMA batch"
            raise UNetTimeoutError(f"unet: a bounded tensor-core wait ran out (flag {f}: {what}); "
                                   "the network's outputs and parameters are invalid")

    def forward(self, ols1, ols2, prev_out, albedo, normal):
        self.raise_if_failed()
        B, H, W, _ = ols1.shape
        ws = self._workspace(B, H, W)
        ins = [t.contiguous() for t in (ols1, ols2, prev_out, albedo, normal)]
        band = torch.empty((B, H, W, 5), dtype=torch.float32, device=self.device)
        alpha = torch.empty((B, H, W, 1), dtype=torch.float32, device=self.device)
        _lib.check(_lib.lib().cd_unet_forward(*[_ptr(t) for t in ins], _ptr(self.params), _ptr(band), _ptr(alpha),
                                              B, H, W, _ptr(ws), ws.numel(), _stream()), "unet_forward")
        return band, alpha

    __call__ = forward

    def backward(self, g_band, g_alpha):
        """dL/dparams (into self.grads) of the last forward."""
        B, H, W = self._shape
        g_band, g_alpha = g_band.contiguous(), g_alpha.contiguous()
        _lib.check(_lib.lib().cd_unet_backward(_ptr(g_band), _ptr(g_alpha), _ptr(self.params), _ptr(self.grads),
                                               B, H, W, _ptr(self.ws), self.ws.numel(), _stream()), "unet_backward")
        return self.grads

    def apply_gradients(self):
        _lib.check(_lib.lib().cd_adam_update(_ptr(self.params), _ptr(self.grads), _ptr(self.m), _ptr(self.v),
                                             self.n, _ptr(self.step), self.lr, BETA1, BETA2, EPSILON, _stream()),
                   "adam_update")

    def on_gradients(self, g_band, g_alpha):
        self.backward(g_band, g_alpha)
        self.apply_gradients()
        if not torch.cuda.is_current_stream_capturing():
            self.enqueue_error_readback()


class UNetTimeoutError(RuntimeError):
    """A bounded wait of the U-Net's tensor-core kernels ran out."""


def to_planes(x):
    """[B,H,W,C] (C a multiple of 8) -> the kernels' row-chunk planes [B,H,C/8,W,8]."""
    B, H, W, C = x.shape
    return x.reshape(B, H, W, C // 8, 8).permute(0, 1, 3, 2, 4).contiguous()


def from_planes(p):
    """Row-chunk planes [B,H,C/8,W,8] -> [B,H,W,C]."""
    B, H, n, W, _ = p.shape
    return p.permute(0, 1, 3, 2, 4).reshape(B, H, W, 8 * n)


def conv3x3(weight, bias, x, cin: int, cout: int, dgrad: bool = False):
    """One 3x3 conv layer on the tensor-core kernel (cd_unet_conv3x3).
    x: [B,H,W,C] bf16 with C = cin (or cout for dgrad) rounded up to 8; the
    kernel reads and writes row-chunk planes, converted here."""
    B, H, W, _ = x.shape
    out_ch = cin if dgrad else cout
    xp = to_planes(x)   # held until the launch is queued
    yp = torch.empty((B, H, (out_ch + 7) // 8, W, 8), dtype=torch.bfloat16, device=x.device)
    L = _lib.lib()
    nb = int(L.cd_unet_conv3x3_workspace_size(cin, cout))
    ws = torch.zeros((max(nb, 1),), dtype=torch.uint8, device=x.device)
    _lib.check(L.cd_unet_conv3x3(_ptr(weight), None if bias is None else _ptr(bias), _ptr(xp), _ptr(yp),
                                 cin, cout, int(dgrad), B, H, W, _ptr(ws), nb, _stream()), "unet_conv3x3")
    return from_planes(yp), ws


def conv3x3_wgrad(x, dz, cin: int, cout: int):
    """[dW (3,3,cin,cout), db (cout,)] of a 3x3 conv layer (cd_unet_conv3x3_wgrad);
    x, dz as for conv3x3."""
    B, H, W, _ = x.shape
    L = _lib.lib()
    nb = int(L.cd_unet_conv3x3_wgrad_workspace_size(cin, cout, B, H, W))
    ws = torch.zeros((max(nb, 1),), dtype=torch.uint8, device=x.device)
    g = torch.empty((9 * cin * cout + cout,), dtype=torch.float32, device=x.device)
    xp, dzp = to_planes(x), to_planes(dz)   # held until the launch is queued
    _lib.check(L.cd_unet_conv3x3_wgrad(_ptr(xp), _ptr(dzp), _ptr(g), cin, cout, B, H, W, _ptr(ws), nb, _stream()),
               "unet_conv3x3_wgrad")
    return g[:9 * cin * cout].view(3, 3, cin, cout), g[9 * cin * cout:], ws
