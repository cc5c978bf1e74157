"""CPU oracle: ctypes wrapper of liboracle.so (cd_oracle.c).

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA kernels and the timed CPU
baseline of bench.py.  Arrays are NHWC float32 numpy arrays; every function
restates the reference op named in its docstring (see cd_oracle.c for the
file:line of each formula).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

# Reprojection rounding mode (cd_oracle.c, orc_reproject): which float
# expressions are fused multiply-adds.  Pinned against the reference kernels'
# own outputs on rounding-boundary inputs (tests/golden/reproject_*.npz):
# pos + mvec*dim is fused, the squared normal distance is
# fma(z, z, fma(x, x, y*y)), the bilinear weight sum adds rounded products.
# (Whether posPrev is fused could not be observed: bilinear reprojection is
# continuous in it; it shares the fused mvec*dim term of the rounded position.)
RP_FMA_IPOS, RP_FMA_POSPREV, RP_FMA_SUMW = 1, 2, 16
RP_DOT_SHIFT = 2
RP_MODE = RP_FMA_IPOS | RP_FMA_POSPREV | (1 << RP_DOT_SHIFT)

_P = ctypes.c_void_p
_I = ctypes.c_int
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        L = ctypes.CDLL(LIB)
        L.orc_variance.argtypes = [_P, _P, _I, _I, _I]
        L.orc_cross_regression.argtypes = [_P] * 10 + [_I] * 6
        L.orc_spatial_filter.argtypes = [_P] * 11 + [_I] * 4
        L.orc_spatial_filter_grad.argtypes = [_P] * 7 + [_I] * 3
        L.orc_reproject.argtypes = [_P, _I, _P, _P, _P] + [_P] * 8 + [_I] * 4
        L.orc_erode3x3.argtypes = [_P, _P, _I, _I, _I]
        L.orc_temporal_screening.argtypes = [_P] * 10 + [_I] * 5
        for f in ("orc_variance", "orc_cross_regression", "orc_spatial_filter",
                  "orc_spatial_filter_grad", "orc_reproject", "orc_erode3x3",
                  "orc_temporal_screening"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def _f32(a, name, ch=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 4 or (ch is not None and a.shape[3] != ch):
        raise ValueError(f"{name}: expected NHWC with {ch} channels, got {a.shape}")
    return a


def _p(a):
    return a.ctypes.data_as(_P)


def variance(img):
    """EstInputVarianceKernel (ops/regression.cu.cc:244-276), win 3."""
    img = _f32(img, "img", 3)
    B, H, W, _ = img.shape
    out = np.empty((B, H, W, 1), np.float32)
    lib().orc_variance(_p(img), _p(out), B, H, W)
    return out


def cross_regression(imga, imgb, albedo, normal, win_size, sparsity, recon_scale=1,
                     return_beta=False):
    """CrossRegressionFunc (ops/regression.cu.cc:477-500) for every batch
    slice: (outa, outb, vara, varb[, betaA, betaB]); beta is
    [B, H/s, W/s, 6, 3] (coefficient, channel)."""
    imga, imgb = _f32(imga, "imga", 3), _f32(imgb, "imgb", 3)
    albedo, normal = _f32(albedo, "albedo", 3), _f32(normal, "normal", 3)
    B, H, W, _ = imga.shape
    s, r = int(sparsity), int(recon_scale)
    outa = np.empty((B, H // r, W // r, 3), np.float32)
    outb = np.empty_like(outa)
    vara = np.empty((B, H, W, 1), np.float32)
    varb = np.empty_like(vara)
    ba = np.empty((B, H // s, W // s, 6, 3), np.float32)
    bb = np.empty_like(ba)
    lib().orc_cross_regression(_p(imga), _p(imgb), _p(albedo), _p(normal), _p(outa), _p(outb),
                               _p(vara), _p(varb), _p(ba), _p(bb), B, H, W, int(win_size), s, r)
    if return_beta:
        return outa, outb, vara, varb, ba, bb
    return outa, outb, vara, varb


def spatial_filter(imga, imgb, albedo, normal, band, win_size, partials=False):
    """SpatialFilterKernel (ops/regression.cu.cc:84-195):
    (acca, accb, wsuma, wsumb[, partA, partB]); partials are [B,H,W,16]."""
    imga, imgb = _f32(imga, "imga", 3), _f32(imgb, "imgb", 3)
    albedo, normal = _f32(albedo, "albedo", 3), _f32(normal, "normal", 3)
    band = _f32(band, "band", 5)
    B, H, W, _ = imga.shape
    acca, accb = np.empty_like(imga), np.empty_like(imga)
    wsa = np.empty((B, H, W, 1), np.float32)
    wsb = np.empty_like(wsa)
    pa = np.empty((B, H, W, 16), np.float32) if partials else None
    pb = np.empty_like(pa) if partials else None
    lib().orc_spatial_filter(_p(imga), _p(imgb), _p(albedo), _p(normal), _p(band), _p(acca),
                             _p(accb), _p(wsa), _p(wsb), _p(pa) if partials else None,
                             _p(pb) if partials else None, B, H, W, int(win_size))
    if partials:
        return acca, accb, wsa, wsb, pa, pb
    return acca, accb, wsa, wsb


def spatial_filter_grad_from_partials(g_acca, g_accb, g_wsa, g_wsb, partA, partB):
    """SpatialFilterGradKernel (ops/regression.cu.cc:33-81)."""
    g_acca, g_accb = _f32(g_acca, "g_acca", 3), _f32(g_accb, "g_accb", 3)
    g_wsa, g_wsb = _f32(g_wsa, "g_wsa", 1), _f32(g_wsb, "g_wsb", 1)
    partA, partB = _f32(partA, "partA", 16), _f32(partB, "partB", 16)
    B, H, W, _ = g_acca.shape
    out = np.empty((B, H, W, 5), np.float32)
    lib().orc_spatial_filter_grad(_p(g_acca), _p(g_accb), _p(g_wsa), _p(g_wsb), _p(partA),
                                  _p(partB), _p(out), B, H, W)
    return out


def spatial_filter_grad(g_acca, g_accb, g_wsa, g_wsb, imga, imgb, albedo, normal, band, win_size):
    """The reference's gradient path: forward storing partials, then the dot."""
    *_, pa, pb = spatial_filter(imga, imgb, albedo, normal, band, win_size, partials=True)
    return spatial_filter_grad_from_partials(g_acca, g_accb, g_wsa, g_wsb, pa, pb)


def reproject(mvec, input_list, linear_z, prev_linear_z, normal, prev_normal, pn_fwidth,
              opacity, prev_opacity, mode=None):
    """Reproject (ops/reproject.cu.cc:32-238): (success bool [B,H,W,1], outputs)."""
    mvec = _f32(mvec, "mvec", 3)
    B, H, W, _ = mvec.shape
    ins = [_f32(t, f"input_list[{i}]") for i, t in enumerate(input_list)]
    outs = [np.empty_like(t) for t in ins]
    n = len(ins)
    arrs = [_f32(linear_z, "linear_z", 3), _f32(prev_linear_z, "prev_linear_z", 3),
            _f32(normal, "normal", 3), _f32(prev_normal, "prev_normal", 3),
            _f32(pn_fwidth, "pn_fwidth", 3), _f32(opacity, "opacity", 1),
            _f32(prev_opacity, "prev_opacity", 1)]
    succ = np.empty((B, H, W, 1), np.uint8)
    in_arr = (_P * n)(*[t.ctypes.data for t in ins])
    out_arr = (_P * n)(*[t.ctypes.data for t in outs])
    ch_arr = (_I * n)(*[t.shape[3] for t in ins])
    lib().orc_reproject(_p(mvec), n, in_arr, ch_arr, out_arr, *[_p(a) for a in arrs], _p(succ),
                        B, H, W, RP_MODE if mode is None else int(mode))
    return succ.astype(bool), outs


def erode3x3(success):
    """tf.nn.erosion2d(SAME, 3x3 ones) + 1 on float(success) (scripts/main.py:270-276)."""
    s = np.ascontiguousarray(success, dtype=np.uint8)
    B, H, W, _ = s.shape
    out = np.empty((B, H, W, 1), np.float32)
    lib().orc_erode3x3(_p(s), _p(out), B, H, W)
    return out


def temporal_screening(c1, c2, prev, prev1, prev2, reproj_success, win_curr, win_prev):
    """TemporalScreening (ops/temporal.cu.cc:57-198): (out, out1, out2, success)."""
    c1, c2 = _f32(c1, "current1", 3), _f32(c2, "current2", 3)
    prev, prev1, prev2 = _f32(prev, "prev", 3), _f32(prev1, "prev1", 3), _f32(prev2, "prev2", 3)
    rs = _f32(reproj_success, "reproj_success", 1)
    B, H, W, _ = c1.shape
    o, o1, o2 = np.empty_like(c1), np.empty_like(c1), np.empty_like(c1)
    sc = np.empty((B, H, W, 1), np.float32)
    lib().orc_temporal_screening(_p(c1), _p(c2), _p(prev), _p(prev1), _p(prev2), _p(rs), _p(o),
                                 _p(o1), _p(o2), _p(sc), B, H, W, int(win_curr), int(win_prev))
    return o, o1, o2, sc
