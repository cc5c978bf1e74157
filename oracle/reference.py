"""The reference's own CUDA kernels, compiled from the reference sources for
sm_100a (oracle/Makefile -> oracle/_ref/libcdref_*.so), called the way its
TensorFlow op wrappers call them.

TEST INFRASTRUCTURE ONLY: the GPU checker for the parity tests, the source
of the golden fixtures (tests/golden/make_golden.py) and the reference arm
of bench.py.  Tensors are torch CUDA tensors, NHWC float32.

Wrapper behaviour replicated from the reference:
  * CrossRegression covers batch slice 0 only (ops/regression.cc:190); its
    coefficient scratch is allocated and zeroed once per shape and then
    reused (ops/regression.cc:138-145, 174-180);
  * SpatialFilter stores the band partials in process-static scratch
    (ops/regression.cc:218-225) and SpatialFilterGrad reads the partials of
    the most recent forward call;
  * Reproject uploads its pointer tables with blocking cudaMemcpy every call
    (ops/reproject.cc:151-153) and launches once per batch slice;
  * TemporalScreening covers batch slice 0 only (ops/temporal.cu.cc:76).
The helpers below loop over batch slices where the reference covers slice 0
only, so they can be compared with the batched ops.
"""
from __future__ import annotations

import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_P = ctypes.c_void_p
_I = ctypes.c_int
_libs = {}
_scratch = {}


def available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f"libcdref_{n}.so"))
               for n in ("regression", "reproject", "temporal"))


def _lib(name):
    if name not in _libs:
        path = os.path.join(REF_DIR, f"libcdref_{name}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle ref` where the "
                                    "reference sources are present")
        L = ctypes.CDLL(path)
        if name == "regression":
            L.cdref_cross_regression.argtypes = [_P] * 10 + [_I] * 5 + [_P]
            L.cdref_spatial_filter.argtypes = [_P] * 11 + [_I] * 3 + [_P]
            L.cdref_spatial_filter_grad.argtypes = [_P] * 12 + [_I] * 3 + [_P]
        elif name == "reproject":
            L.cdref_reproject.argtypes = [_P, _I, _P, _P, _P] + [_P] * 8 + [_I] * 3 + [_P]
        else:
            L.cdref_temporal_screening.argtypes = [_P] * 10 + [_I] * 4 + [_P]
        _libs[name] = L
    return _libs[name]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _st():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference {what} failed with cudaError {rc}")


def _zeros_once(key, shape, device):
    t = _scratch.get(key)
    if t is None or t.device != device:
        t = torch.zeros(shape, dtype=torch.float32, device=device)
        _scratch[key] = t
    return t


def cross_regression(imga, imgb, albedo, normal, win_size, sparsity, recon_scale=1):
    B, H, W, _ = imga.shape
    s, r = int(sparsity), int(recon_scale)
    dev = imga.device
    ba = _zeros_once(("betaA", H, W, s), (H // s, W // s, 24), dev)
    bb = _zeros_once(("betaB", H, W, s), (H // s, W // s, 24), dev)
    outa = torch.empty((B, H // r, W // r, 3), dtype=torch.float32, device=dev)
    outb = torch.empty_like(outa)
    vara = torch.empty((B, H, W, 1), dtype=torch.float32, device=dev)
    varb = torch.empty_like(vara)
    L = _lib("regression")
    for b in range(B):
        _ok(L.cdref_cross_regression(_p(imga[b]), _p(imgb[b]), _p(albedo[b]), _p(normal[b]),
                                     _p(outa[b]), _p(outb[b]), _p(vara[b]), _p(varb[b]),
                                     _p(ba), _p(bb), H, W, int(win_size), s, r, _st()),
            "CrossRegression")
    return outa, outb, vara, varb


def spatial_filter(imga, imgb, albedo, normal, band, win_size):
    """Forward; leaves the band partials of every slice in the static scratch."""
    B, H, W, _ = imga.shape
    dev = imga.device
    pa = _zeros_once(("gradBandA", B, H, W), (B, H, W, 16), dev)
    pb = _zeros_once(("gradBandB", B, H, W), (B, H, W, 16), dev)
    _scratch["last_partials"] = (pa, pb)
    acca, accb = torch.empty_like(imga), torch.empty_like(imga)
    wsa = torch.empty((B, H, W, 1), dtype=torch.float32, device=dev)
    wsb = torch.empty_like(wsa)
    L = _lib("regression")
    for b in range(B):
        _ok(L.cdref_spatial_filter(_p(imga[b]), _p(imgb[b]), _p(albedo[b]), _p(normal[b]),
                                   _p(band[b]), _p(acca[b]), _p(accb[b]), _p(wsa[b]), _p(wsb[b]),
                                   _p(pa[b]), _p(pb[b]), H, W, int(win_size), _st()),
            "SpatialFilter")
    return acca, accb, wsa, wsb


def spatial_filter_grad(g_acca, g_accb, g_wsa, g_wsb, imga, imgb, albedo, normal, band, win_size):
    """Gradient from the partials of the most recent spatial_filter call."""
    B, H, W, _ = imga.shape
    pa, pb = _scratch["last_partials"]
    out = torch.empty((B, H, W, 5), dtype=torch.float32, device=imga.device)
    L = _lib("regression")
    for b in range(B):
        _ok(L.cdref_spatial_filter_grad(_p(g_acca[b]), _p(g_accb[b]), _p(g_wsa[b]), _p(g_wsb[b]),
                                        _p(imga[b]), _p(imgb[b]), _p(albedo[b]), _p(normal[b]),
                                        _p(band[b]), _p(out[b]), _p(pa[b]), _p(pb[b]), H, W,
                                        int(win_size), _st()), "SpatialFilterGrad")
    return out


def reproject(mvec, input_list, linear_z, prev_linear_z, normal, prev_normal, pn_fwidth,
              opacity, prev_opacity):
    B, H, W, _ = mvec.shape
    n = len(input_list)
    outs = [torch.empty_like(t) for t in input_list]
    succ = torch.empty((B, H, W, 1), dtype=torch.bool, device=mvec.device)
    in_arr = (_P * n)(*[t.data_ptr() for t in input_list])
    out_arr = (_P * n)(*[t.data_ptr() for t in outs])
    ch_arr = (_I * n)(*[int(t.shape[3]) for t in input_list])
    _ok(_lib("reproject").cdref_reproject(
        _p(mvec), n, in_arr, ch_arr, out_arr, _p(linear_z), _p(prev_linear_z), _p(normal),
        _p(prev_normal), _p(pn_fwidth), _p(opacity), _p(prev_opacity), _p(succ), B, H, W, _st()),
        "Reproject")
    return succ, outs


def erode3x3(success):
    """Stand-in for TensorFlow's builtin erosion2d(SAME) + 1 (not part of the
    reference's own code): min over the in-bounds 3x3 window."""
    x = success.float().permute(0, 3, 1, 2)
    return (-torch.nn.functional.max_pool2d(-x, 3, stride=1, padding=1)).permute(0, 2, 3, 1).contiguous()


def temporal_screening(c1, c2, prev, prev1, prev2, reproj_success, win_curr, win_prev):
    B, H, W, _ = c1.shape
    o, o1, o2 = (torch.empty_like(c1) for _ in range(3))
    sc = torch.empty((B, H, W, 1), dtype=torch.float32, device=c1.device)
    L = _lib("temporal")
    for b in range(B):
        _ok(L.cdref_temporal_screening(_p(c1[b]), _p(c2[b]), _p(prev[b]), _p(prev1[b]),
                                       _p(prev2[b]), _p(reproj_success[b]), _p(o[b]), _p(o1[b]),
                                       _p(o2[b]), _p(sc[b]), H, W, int(win_curr), int(win_prev),
                                       _st()), "TemporalScreening")
    return o, o1, o2, sc
