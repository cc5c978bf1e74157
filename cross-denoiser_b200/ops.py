"""Drop-in op surface of the reference's scripts/ops.py, on sm_100a kernels.

Same op names, argument order, keyword attributes, NHWC float32 layouts and
output tuples as the TensorFlow custom ops the reference loads
(scripts/ops.py:18-40; schemas in ops/regression.cc:25-103,
ops/reproject.cc:34-69, ops/temporal.cu.cc:263-285).  Tensors are PyTorch
CUDA tensors; every op runs on the current CUDA stream through the C ABI of
include/cd_ops.h.  Invalid arguments raise ValueError, the analogue of the
reference's InvalidArgument errors.

Differences from the reference, all deliberate:
  * every op processes all B batch slices (the reference covers slice 0 only
    in CrossRegression, SpatialFilter and TemporalScreening), and the
    variance outputs of cross_regression are [B,H,W,1] instead of [1,H,W,1];
  * spatial_filter_grad recomputes the filter weights from the inputs the
    reference passes to it (it reads them instead of process-static partials
    stored by the last forward call), so it is stateless and re-entrant;
  * shapes on which the reference kernels index out of bounds are rejected.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import torch

from . import _lib

__all__ = [
    "cross_regression", "spatial_filter", "spatial_filter_grad", "temporal_screening",
    "Reproject", "reproject", "erode3x3", "erode_temporal_screening", "prepare_input",
    "aggregation_loss", "filter_aggregate",
]


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _img(t: torch.Tensor, name: str, channels: int | None, ref: torch.Tensor | None = None,
         dtype=torch.float32) -> torch.Tensor:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (the ops have no CPU path)")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if t.dim() != 4:
        raise ValueError(f"{name} must be NHWC (rank 4), got shape {tuple(t.shape)}")
    if channels is not None and t.shape[3] != channels:
        raise ValueError(f"{name} must have {channels} channels, got {t.shape[3]}")
    if ref is not None:
        if tuple(t.shape[:3]) != tuple(ref.shape[:3]):
            raise ValueError(f"{name} has shape {tuple(t.shape)}, expected [B,H,W] = {tuple(ref.shape[:3])}")
        if t.device != ref.device:
            raise ValueError(f"{name} is on {t.device}, expected {ref.device}")
    return t.contiguous()


# ---------------------------------------------------------------------------
# CrossRegression
# ---------------------------------------------------------------------------
def _regression_args(imga, imgb, albedo, normal, win_size, sparsity, recon_scale):
    imga = _img(imga, "imga", 3)
    imgb = _img(imgb, "imgb", 3, imga)
    albedo = _img(albedo, "albedo", 3, imga)
    normal = _img(normal, "normal", 3, imga)
    rs = int(recon_scale)
    if int(win_size) < 1 or int(sparsity) < 1 or rs < 1:
        raise ValueError("win_size, sparsity and recon_scale must be >= 1")
    if rs > int(sparsity):
        raise ValueError("recon_scale must be less than or equal to sparsity")
    B, H, W, _ = imga.shape
    if H % rs or W % rs:
        raise ValueError("Image height and width must be divisible by recon_scale")
    return imga, imgb, albedo, normal, rs


def _cross_regression_raw(imga, imgb, albedo, normal, win_size, sparsity, recon_scale, fp64_cond_limit=0.0,
                          fallback_count=None):
    imga, imgb, albedo, normal, rs = _regression_args(imga, imgb, albedo, normal, win_size, sparsity,
                                                      recon_scale)
    B, H, W, _ = imga.shape
    L = _lib.lib()
    outa = torch.empty((B, H // rs, W // rs, 3), dtype=torch.float32, device=imga.device)
    outb = torch.empty_like(outa)
    vara = torch.empty((B, H, W, 1), dtype=torch.float32, device=imga.device)
    varb = torch.empty_like(vara)
    nbytes = L.cd_cross_regression_workspace_size(B, H, W, int(sparsity))
    ws = torch.empty((max(nbytes, 1),), dtype=torch.uint8, device=imga.device)
    common = (_ptr(imga), _ptr(imgb), _ptr(albedo), _ptr(normal), _ptr(outa), _ptr(outb), _ptr(vara), _ptr(varb),
              B, H, W, int(win_size), int(sparsity), rs)
    if fp64_cond_limit and fp64_cond_limit > 0:
        if fallback_count is not None and (fallback_count.dtype != torch.int32 or not fallback_count.is_cuda):
            raise ValueError("fallback_count must be a CUDA int32 tensor")
        _lib.check(L.cd_cross_regression_fp64_fallback(*common, float(fp64_cond_limit),
                                                       None if fallback_count is None else _ptr(fallback_count),
                                                       _ptr(ws), nbytes, _stream()), "cross_regression_fp64_fallback")
    else:
        _lib.check(L.cd_cross_regression(*common, _ptr(ws), nbytes, _stream()), "cross_regression")
    return outa, outb, vara, varb


def cross_regression_grad(grad_outa, grad_outb, grad_vara, grad_varb, imga, imgb, albedo, normal,
                          win_size: int, sparsity: int, recon_scale: int = 1, _kept=None):
    """(grad_imga, grad_imgb, grad_albedo, grad_normal) of CrossRegression.

    No counterpart in the reference, which registers a gradient only for
    SpatialFilter (scripts/ops.py:23-32).  The analytic derivative of the
    forward above; grad_vara / grad_varb may be None.  The forward is
    recomputed, so only its inputs are needed (cross_regression_grad_kept
    reuses a kept forward instead).
    """
    imga, imgb, albedo, normal, rs = _regression_args(imga, imgb, albedo, normal, win_size, sparsity,
                                                      recon_scale)
    B, H, W, _ = imga.shape
    gshape = (B, H // rs, W // rs, 3)
    grad_outa = _img(grad_outa, "grad_outa", 3)
    grad_outb = _img(grad_outb, "grad_outb", 3, grad_outa)
    if tuple(grad_outa.shape) != gshape:
        raise ValueError(f"grad_outa must have shape {gshape}, got {tuple(grad_outa.shape)}")
    gv = []
    for g, nm in ((grad_vara, "grad_vara"), (grad_varb, "grad_varb")):
        if g is not None:
            g = _img(g, nm, 1)
            if tuple(g.shape) != (B, H, W, 1):
                raise ValueError(f"{nm} must have shape {(B, H, W, 1)}, got {tuple(g.shape)}")
        gv.append(g)
    L = _lib.lib()
    outs = [torch.empty_like(imga) for _ in range(4)]
    nbytes = L.cd_cross_regression_grad_workspace_size(B, H, W, int(sparsity), rs)
    if _kept is None:
        ws, fn, name = torch.empty((max(nbytes, 1),), dtype=torch.uint8, device=imga.device), \
            L.cd_cross_regression_grad, "cross_regression_grad"
    else:
        if _kept.dtype != torch.uint8 or _kept.numel() < nbytes or _kept.device != imga.device:
            raise ValueError(f"workspace must be a uint8 tensor of >= {nbytes} bytes on {imga.device}")
        ws, fn, name = _kept, L.cd_cross_regression_grad_kept, "cross_regression_grad_kept"
    _lib.check(fn(
        _ptr(imga), _ptr(imgb), _ptr(albedo), _ptr(normal), _ptr(grad_outa), _ptr(grad_outb),
        None if gv[0] is None else _ptr(gv[0]), None if gv[1] is None else _ptr(gv[1]),
        *[_ptr(o) for o in outs], B, H, W, int(win_size), int(sparsity), rs, _ptr(ws), ws.numel(),
        _stream()), name)
    return tuple(outs)


def cross_regression_keep(imga, imgb, albedo, normal, win_size: int, sparsity: int, recon_scale: int = 1):
    """cross_regression's four outputs (bit-identical) and a workspace that
    keeps the forward's variances, coefficients and Cholesky factors for
    cross_regression_grad_kept (cd_cross_regression_keep).  No counterpart in
    the reference.  Returns ((outa, outb, out_vara, out_varb), workspace)."""
    imga, imgb, albedo, normal, rs = _regression_args(imga, imgb, albedo, normal, win_size, sparsity,
                                                      recon_scale)
    B, H, W, _ = imga.shape
    outa = imga.new_empty((B, H // rs, W // rs, 3))
    outb = imga.new_empty((B, H // rs, W // rs, 3))
    vara = imga.new_empty((B, H, W, 1))
    varb = imga.new_empty((B, H, W, 1))
    L = _lib.lib()
    nbytes = L.cd_cross_regression_grad_workspace_size(B, H, W, int(sparsity), rs)
    ws = torch.empty((max(nbytes, 1),), dtype=torch.uint8, device=imga.device)
    _lib.check(L.cd_cross_regression_keep(_ptr(imga), _ptr(imgb), _ptr(albedo), _ptr(normal), _ptr(outa),
                                          _ptr(outb), _ptr(vara), _ptr(varb), B, H, W, int(win_size),
                                          int(sparsity), rs, _ptr(ws), nbytes, _stream()),
               "cross_regression_keep")
    return (outa, outb, vara, varb), ws


def cross_regression_grad_kept(grad_outa, grad_outb, grad_vara, grad_varb, imga, imgb, albedo, normal,
                               win_size: int, sparsity: int, recon_scale: int, workspace: torch.Tensor):
    """cross_regression_grad's result (bit-identical) from the workspace of
    cross_regression_keep on the same inputs, without recomputing the
    forward (cd_cross_regression_grad_kept)."""
    return cross_regression_grad(grad_outa, grad_outb, grad_vara, grad_varb, imga, imgb, albedo, normal,
                                 win_size, sparsity, recon_scale, _kept=workspace)


class _CrossRegressionFn(torch.autograd.Function):
    """Autograd wrapper: forward cd_cross_regression_keep, backward
    cd_cross_regression_grad_kept on the kept workspace."""

    @staticmethod
    def forward(ctx, imga, imgb, albedo, normal, win_size, sparsity, recon_scale):
        outs, ws = cross_regression_keep(imga, imgb, albedo, normal, win_size, sparsity, recon_scale)
        ctx.save_for_backward(imga, imgb, albedo, normal)
        ctx.attrs = (int(win_size), int(sparsity), int(recon_scale))
        ctx.ws = ws
        return outs

    @staticmethod
    def backward(ctx, g_outa, g_outb, g_vara, g_varb):
        imga, imgb, albedo, normal = ctx.saved_tensors
        B, H, W, _ = imga.shape
        rs = ctx.attrs[2]
        if g_outa is None:
            g_outa = imga.new_zeros((B, H // rs, W // rs, 3))
        if g_outb is None:
            g_outb = imga.new_zeros((B, H // rs, W // rs, 3))
        grads = cross_regression_grad_kept(g_outa, g_outb, g_vara, g_varb, imga, imgb, albedo, normal,
                                           *ctx.attrs, ctx.ws)
        ctx.ws = None
        return (*grads, None, None, None)


def cross_regression(imga, imgb, albedo, normal, win_size: int, sparsity: int,
                     recon_scale: int = 1, name=None, fp64_cond_limit: float = 0.0, fallback_count=None):
    """(outa, outb, out_vara, out_varb) = cross_regression(imga, imgb, albedo, normal, ...).

    Reference: REGISTER_OP("CrossRegression") ops/regression.cc:25-57 and
    CrossRegressionFunc ops/regression.cu.cc:477-500.  outa is imgb predicted
    from imga's features, outb imga from imgb's; out_vara/out_varb are the
    3x3 variance estimates of imga/imgb.  Differentiable with respect to the
    four images through cross_regression_grad when any of them requires grad.

    fp64_cond_limit > 0 (not in the reference) re-solves, in double, every
    centre whose FP32 Cholesky pivots give a condition estimate above it and
    adds the number of such (centre, channel) solves to `fallback_count` (a
    CUDA int32 tensor) when given.
    """
    if torch.is_grad_enabled() and any(isinstance(t, torch.Tensor) and t.requires_grad
                                       for t in (imga, imgb, albedo, normal)):
        return _CrossRegressionFn.apply(imga, imgb, albedo, normal, int(win_size), int(sparsity),
                                        int(recon_scale))
    return _cross_regression_raw(imga, imgb, albedo, normal, win_size, sparsity, recon_scale, fp64_cond_limit,
                                 fallback_count)


# ---------------------------------------------------------------------------
# SpatialFilter and its gradient
# ---------------------------------------------------------------------------
def _spatial_filter_raw(imga, imgb, albedo, normal, band, win_size):
    imga = _img(imga, "imga", 3)
    imgb = _img(imgb, "imgb", 3, imga)
    albedo = _img(albedo, "albedo", 3, imga)
    normal = _img(normal, "normal", 3, imga)
    band = _img(band, "band", 5, imga)
    B, H, W, _ = imga.shape
    acca = torch.empty_like(imga)
    accb = torch.empty_like(imga)
    wsa = torch.empty((B, H, W, 1), dtype=torch.float32, device=imga.device)
    wsb = torch.empty_like(wsa)
    _lib.check(_lib.lib().cd_spatial_filter(_ptr(imga), _ptr(imgb), _ptr(albedo), _ptr(normal),
                                            _ptr(band), _ptr(acca), _ptr(accb), _ptr(wsa),
                                            _ptr(wsb), B, H, W, int(win_size), _stream()),
               "spatial_filter")
    return acca, accb, wsa, wsb


def spatial_filter_grad(grad_acca, grad_accb, grad_wgtsuma, grad_wgtsumb, imga, imgb,
                        img_albedo, img_normal, band, win_size: int, name=None):
    """out_grad_band = spatial_filter_grad(...), schema ops/regression.cc:88-103.

    Gradient of the spatial filter's four outputs with respect to band
    (channel 0 from buffer A, 1 from B, 2..4 from both), as
    SpatialFilterGradKernel ops/regression.cu.cc:33-81 computes it; the
    weights are recomputed from imga/imgb/img_albedo/img_normal/band.
    """
    imga = _img(imga, "imga", 3)
    imgb = _img(imgb, "imgb", 3, imga)
    img_albedo = _img(img_albedo, "img_albedo", 3, imga)
    img_normal = _img(img_normal, "img_normal", 3, imga)
    band = _img(band, "band", 5, imga)
    ga = _img(grad_acca, "grad_acca", 3, imga)
    gb = _img(grad_accb, "grad_accb", 3, imga)
    gwa = _img(grad_wgtsuma, "grad_wgtsuma", 1, imga)
    gwb = _img(grad_wgtsumb, "grad_wgtsumb", 1, imga)
    B, H, W, _ = imga.shape
    out = torch.empty_like(band)
    _lib.check(_lib.lib().cd_spatial_filter_grad(_ptr(ga), _ptr(gb), _ptr(gwa), _ptr(gwb),
                                                 _ptr(imga), _ptr(imgb), _ptr(img_albedo),
                                                 _ptr(img_normal), _ptr(band), _ptr(out),
                                                 B, H, W, int(win_size), _stream()),
               "spatial_filter_grad")
    return out


class _SpatialFilterFn(torch.autograd.Function):
    """Autograd wrapper with the reference's registered gradient
    (scripts/ops.py:23-32): a gradient for band only, None for the images."""

    @staticmethod
    def forward(ctx, imga, imgb, albedo, normal, band, win_size):
        outs = _spatial_filter_raw(imga, imgb, albedo, normal, band, win_size)
        ctx.save_for_backward(imga, imgb, albedo, normal, band)
        ctx.win_size = int(win_size)
        return outs

    @staticmethod
    def backward(ctx, g_acca, g_accb, g_wsa, g_wsb):
        imga, imgb, albedo, normal, band = ctx.saved_tensors
        def z(g, like):
            return torch.zeros_like(like) if g is None else g
        B, H, W, _ = imga.shape
        w1 = imga.new_empty((B, H, W, 1))
        gband = spatial_filter_grad(z(g_acca, imga), z(g_accb, imga), z(g_wsa, w1), z(g_wsb, w1),
                                    imga, imgb, albedo, normal, band, ctx.win_size)
        return None, None, None, None, gband, None


def spatial_filter(imga, imgb, albedo, normal, band, win_size: int, name=None):
    """(out_acca, out_accb, out_wgtsuma, out_wgtsumb) = spatial_filter(...).

    Reference: REGISTER_OP("SpatialFilter") ops/regression.cc:59-86 and
    SpatialFilterKernel ops/regression.cu.cc:84-195.  Differentiable with
    respect to band through spatial_filter_grad.
    """
    if torch.is_grad_enabled() and band.requires_grad:
        return _SpatialFilterFn.apply(imga, imgb, albedo, normal, band, int(win_size))
    return _spatial_filter_raw(imga, imgb, albedo, normal, band, win_size)


def spatial_filter_stored(imga, imgb, albedo, normal, band, win_size: int):
    """(out_acca, out_accb, out_wgtsuma, out_wgtsumb, partials): the forward of
    the reference's design, which keeps the band partials ([B,H,W,32] floats,
    ops/regression.cc:218-225) for the gradient; see spatial_filter_grad_stored.
    Same outputs as spatial_filter."""
    imga = _img(imga, "imga", 3)
    imgb = _img(imgb, "imgb", 3, imga)
    albedo = _img(albedo, "albedo", 3, imga)
    normal = _img(normal, "normal", 3, imga)
    band = _img(band, "band", 5, imga)
    B, H, W, _ = imga.shape
    acca, accb = torch.empty_like(imga), torch.empty_like(imga)
    wsa = imga.new_empty((B, H, W, 1))
    wsb = torch.empty_like(wsa)
    part = imga.new_empty((B, H, W, 32))
    _lib.check(_lib.lib().cd_spatial_filter_stored(_ptr(imga), _ptr(imgb), _ptr(albedo), _ptr(normal), _ptr(band),
                                                   _ptr(acca), _ptr(accb), _ptr(wsa), _ptr(wsb), _ptr(part), B, H,
                                                   W, int(win_size), _stream()), "spatial_filter_stored")
    return acca, accb, wsa, wsb, part


def spatial_filter_grad_stored(grad_acca, grad_accb, grad_wgtsuma, grad_wgtsumb, partials):
    """dL/dband from the partials stored by spatial_filter_stored (the
    reference's SpatialFilterGradKernel data flow); equals spatial_filter_grad."""
    ga = _img(grad_acca, "grad_acca", 3)
    gb = _img(grad_accb, "grad_accb", 3, ga)
    gwa = _img(grad_wgtsuma, "grad_wgtsuma", 1, ga)
    gwb = _img(grad_wgtsumb, "grad_wgtsumb", 1, ga)
    part = _img(partials, "partials", 32, ga)
    B, H, W, _ = ga.shape
    out = ga.new_empty((B, H, W, 5))
    _lib.check(_lib.lib().cd_spatial_filter_grad_stored(_ptr(ga), _ptr(gb), _ptr(gwa), _ptr(gwb), _ptr(part),
                                                        _ptr(out), B, H, W, _stream()), "spatial_filter_grad_stored")
    return out


# ---------------------------------------------------------------------------
# Reproject
# ---------------------------------------------------------------------------
def reproject(mvec, input_list: Sequence[torch.Tensor], linear_z, prev_linear_z, normal,
              prev_normal, pn_fwidth, opacity, prev_opacity, name=None
              ) -> Tuple[torch.Tensor, List[torch.Tensor]]:
    """(success, output_list) = Reproject(mvec, input_list, ...).

    Reference: REGISTER_OP("Reproject") ops/reproject.cc:34-69 and the
    Reproject kernel ops/reproject.cu.cc:53-238.  success is a bool tensor
    [B,H,W,1]; output_list holds one reprojected tensor per input.
    """
    mvec = _img(mvec, "mvec", 3)
    linear_z = _img(linear_z, "linear_z", 3, mvec)
    prev_linear_z = _img(prev_linear_z, "prev_linear_z", 3, mvec)
    normal = _img(normal, "normal", 3, mvec)
    prev_normal = _img(prev_normal, "prev_normal", 3, mvec)
    pn_fwidth = _img(pn_fwidth, "pn_fwidth", 3, mvec)
    opacity = _img(opacity, "opacity", 1, mvec)
    prev_opacity = _img(prev_opacity, "prev_opacity", 1, mvec)
    inputs = [_img(t, f"input_list[{i}]", None, mvec) for i, t in enumerate(input_list)]
    n = len(inputs)
    if n < 1 or n > _lib.REPROJECT_MAX_LIST:
        raise ValueError(f"input_list must hold 1..{_lib.REPROJECT_MAX_LIST} tensors")
    B, H, W, _ = mvec.shape
    outputs = [torch.empty_like(t) for t in inputs]
    success = torch.empty((B, H, W, 1), dtype=torch.bool, device=mvec.device)
    in_arr = (ctypes.c_void_p * n)(*[t.data_ptr() for t in inputs])
    out_arr = (ctypes.c_void_p * n)(*[t.data_ptr() for t in outputs])
    ch_arr = (ctypes.c_int * n)(*[int(t.shape[3]) for t in inputs])
    _lib.check(_lib.lib().cd_reproject(_ptr(mvec), n, in_arr, ch_arr, out_arr, _ptr(linear_z),
                                       _ptr(prev_linear_z), _ptr(normal), _ptr(prev_normal),
                                       _ptr(pn_fwidth), _ptr(opacity), _ptr(prev_opacity),
                                       _ptr(success), B, H, W, _stream()), "reproject",
               kernels=2 if n == 3 and all(int(t.shape[3]) == 3 for t in inputs) else 1)
    return success, outputs


Reproject = reproject


# ---------------------------------------------------------------------------
# Erosion and temporal screening
# ---------------------------------------------------------------------------
def erode3x3(success):
    """float 3x3 erosion of a bool mask with SAME padding; the
    tf.nn.erosion2d(...) + 1 of scripts/main.py:270-276."""
    success = _img(success, "success", 1, dtype=torch.bool)
    B, H, W, _ = success.shape
    out = torch.empty(success.shape, dtype=torch.float32, device=success.device)
    _lib.check(_lib.lib().cd_erode3x3(_ptr(success), _ptr(out), B, H, W, _stream()), "erode3x3")
    return out


def temporal_screening(current1, current2, prev, prev1, prev2, reproj_success,
                       win_curr: int, win_prev: int, name=None):
    """(output, output1, output2, success) = temporal_screening(...).

    Reference: REGISTER_OP("TemporalScreening") ops/temporal.cu.cc:263-285
    and the TemporalScreening kernel :57-198.
    """
    current1 = _img(current1, "current1", 3)
    current2 = _img(current2, "current2", 3, current1)
    prev = _img(prev, "prev", 3, current1)
    prev1 = _img(prev1, "prev1", 3, current1)
    prev2 = _img(prev2, "prev2", 3, current1)
    reproj_success = _img(reproj_success, "reproj_success", 1, current1)
    B, H, W, _ = current1.shape
    out, out1, out2 = (torch.empty_like(current1) for _ in range(3))
    succ = torch.empty_like(reproj_success)
    _lib.check(_lib.lib().cd_temporal_screening(
        _ptr(current1), _ptr(current2), _ptr(prev), _ptr(prev1), _ptr(prev2), _ptr(reproj_success),
        _ptr(out), _ptr(out1), _ptr(out2), _ptr(succ), B, H, W, int(win_curr), int(win_prev),
        _stream()), "temporal_screening")
    return out, out1, out2, succ


def erode_temporal_screening(current1, current2, prev, prev1, prev2, reproj_mask,
                             win_curr: int, win_prev: int):
    """Fused erode3x3 + temporal_screening on the bool reprojection mask.

    Returns (output, output1, output2, success, eroded); identical to
    ``temporal_screening(..., erode3x3(reproj_mask), ...)`` plus the eroded mask.
    """
    current1 = _img(current1, "current1", 3)
    current2 = _img(current2, "current2", 3, current1)
    prev = _img(prev, "prev", 3, current1)
    prev1 = _img(prev1, "prev1", 3, current1)
    prev2 = _img(prev2, "prev2", 3, current1)
    reproj_mask = _img(reproj_mask, "reproj_mask", 1, current1, dtype=torch.bool)
    B, H, W, _ = current1.shape
    out, out1, out2 = (torch.empty_like(current1) for _ in range(3))
    succ = current1.new_empty((B, H, W, 1))
    eroded = torch.empty_like(succ)
    _lib.check(_lib.lib().cd_erode_temporal_screening(
        _ptr(current1), _ptr(current2), _ptr(prev), _ptr(prev1), _ptr(prev2), _ptr(reproj_mask),
        _ptr(eroded), _ptr(out), _ptr(out1), _ptr(out2), _ptr(succ), B, H, W, int(win_curr),
        int(win_prev), _stream()), "erode_temporal_screening")
    return out, out1, out2, succ, eroded


# ---------------------------------------------------------------------------
# The rest of the per-frame step: input preparation and the aggregation loss
# ---------------------------------------------------------------------------
def prepare_input(color, color2):
    """(y1, y2) = (log1p(color), log1p(color2)): prepare_input of
    scripts/main.py:207-212."""
    color = _img(color, "color", 3)
    color2 = _img(color2, "color2", 3, color)
    y1, y2 = torch.empty_like(color), torch.empty_like(color2)
    _lib.check(_lib.lib().cd_prepare_input(_ptr(color), _ptr(color2), _ptr(y1), _ptr(y2), color.numel(),
                                           _stream()), "prepare_input")
    return y1, y2


def _ws(nbytes, device):
    return torch.empty((max(int(nbytes), 4),), dtype=torch.uint8, device=device)


def aggregation_loss(sum1, sumw1, sum2, sumw2, alpha, success, success_prev, prev_out, opacity, label1,
                     label2, prev_label1, prev_label2, with_loss: bool = True):
    """aggregation_loss of scripts/main.py:214-248 with its gradient.

    Returns (out_log, out, loss, avg_loss, grad_sum1, grad_sumw1, grad_sum2,
    grad_sumw2, grad_alpha); ``out_log`` is the reference's ``out`` (log
    domain), ``out`` its max(0, expm1(.)), the gradients are dL/d(input) of
    L = avg_loss.  ``loss`` is None when ``with_loss`` is False.
    """
    sum1 = _img(sum1, "sum1", 3)
    ref = sum1
    sumw1, sum2, sumw2 = _img(sumw1, "sumw1", 1, ref), _img(sum2, "sum2", 3, ref), _img(sumw2, "sumw2", 1, ref)
    alpha, success = _img(alpha, "alpha", 1, ref), _img(success, "success", 1, ref)
    success_prev, prev_out = _img(success_prev, "success_prev", 1, ref), _img(prev_out, "prev_out", 3, ref)
    opacity = _img(opacity, "opacity", 1, ref)
    labels = [_img(t, n, 3, ref) for t, n in ((label1, "label1"), (label2, "label2"),
                                                (prev_label1, "prev_label1"), (prev_label2, "prev_label2"))]
    B, H, W, _ = sum1.shape
    out_log, out = torch.empty_like(sum1), torch.empty_like(sum1)
    loss = torch.empty_like(sum1) if with_loss else None
    avg = sum1.new_empty(())
    g1, g2 = torch.empty_like(sum1), torch.empty_like(sum1)
    gw1, gw2, ga = torch.empty_like(sumw1), torch.empty_like(sumw1), torch.empty_like(sumw1)
    L = _lib.lib()
    nbytes = L.cd_aggregation_workspace_size(B, H, W)
    ws = _ws(nbytes, sum1.device)
    _lib.check(L.cd_aggregation_loss(_ptr(sum1), _ptr(sumw1), _ptr(sum2), _ptr(sumw2), _ptr(alpha), _ptr(success),
                                     _ptr(success_prev), _ptr(prev_out), _ptr(opacity), *[_ptr(t) for t in labels],
                                     _ptr(out_log), _ptr(out), _ptr(loss) if with_loss else None, _ptr(avg),
                                     _ptr(g1), _ptr(gw1), _ptr(g2), _ptr(gw2), _ptr(ga), B, H, W, _ptr(ws),
                                     nbytes, _stream()), "aggregation_loss")
    return out_log, out, loss, avg, g1, gw1, g2, gw2, ga


def filter_aggregate(ols1, ols2, albedo, normal, band, alpha, success, success_prev, prev_out, opacity,
                     prev_ols1, prev_ols2, win_size: int):
    """spatial_filter -> aggregation_loss -> spatial_filter_grad
    (scripts/main.py:295-302) in one kernel pass.

    Returns (out_log, out, avg_loss, grad_band, grad_alpha).
    """
    ols1 = _img(ols1, "ols1", 3)
    ref = ols1
    ols2, albedo, normal = _img(ols2, "ols2", 3, ref), _img(albedo, "albedo", 3, ref), _img(normal, "normal", 3, ref)
    band, alpha = _img(band, "band", 5, ref), _img(alpha, "alpha", 1, ref)
    success, success_prev = _img(success, "success", 1, ref), _img(success_prev, "success_prev", 1, ref)
    prev_out, opacity = _img(prev_out, "prev_out", 3, ref), _img(opacity, "opacity", 1, ref)
    prev_ols1, prev_ols2 = _img(prev_ols1, "prev_ols1", 3, ref), _img(prev_ols2, "prev_ols2", 3, ref)
    B, H, W, _ = ols1.shape
    out_log, out = torch.empty_like(ols1), torch.empty_like(ols1)
    avg = ols1.new_empty(())
    gband, galpha = torch.empty_like(band), torch.empty_like(alpha)
    L = _lib.lib()
    nbytes = L.cd_filter_aggregate_workspace_size(B, H, W)
    ws = _ws(nbytes, ols1.device)
    _lib.check(L.cd_filter_aggregate(_ptr(ols1), _ptr(ols2), _ptr(albedo), _ptr(normal), _ptr(band), _ptr(alpha),
                                     _ptr(success), _ptr(success_prev), _ptr(prev_out), _ptr(opacity),
                                     _ptr(prev_ols1), _ptr(prev_ols2), _ptr(out_log), _ptr(out), _ptr(avg),
                                     _ptr(gband), _ptr(galpha), B, H, W, int(win_size), _ptr(ws), nbytes,
                                     _stream()), "filter_aggregate")
    return out_log, out, avg, gband, galpha
