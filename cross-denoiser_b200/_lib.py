"""ctypes binding of libcdops.so, the C ABI declared in include/cd_ops.h.

The library is built in-tree (``__graft_entry__.build()`` or ``make -C
cross-denoiser_b200/csrc``).  There is no fallback: if the shared object is
missing, :func:`lib` raises, so no op can silently run anywhere but on the
sm_100a kernels.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcdops.so")

CD_OK, CD_EINVAL, CD_ECUDA, CD_ENOMEM = 0, 1, 2, 3
REPROJECT_MAX_LIST = 8

_P = ctypes.c_void_p
_I = ctypes.c_int
_S = ctypes.c_size_t
_F = ctypes.c_float

# name -> (restype, argtypes); mirrors include/cd_ops.h
SIGNATURES = {
    "cd_abi_version": (_I, []),
    "cd_get_last_error": (ctypes.c_char_p, []),
    "cd_cross_regression_workspace_size": (_S, [_I, _I, _I, _I]),
    "cd_cross_regression": (_I, [_P] * 8 + [_I] * 6 + [_P, _S, _P]),
    "cd_cross_regression_fp64_fallback": (_I, [_P] * 8 + [_I] * 6 + [_F, _P, _P, _S, _P]),
    "cd_cross_regression_grad_workspace_size": (_S, [_I] * 5),
    "cd_cross_regression_grad": (_I, [_P] * 12 + [_I] * 6 + [_P, _S, _P]),
    "cd_cross_regression_keep": (_I, [_P] * 8 + [_I] * 6 + [_P, _S, _P]),
    "cd_cross_regression_grad_kept": (_I, [_P] * 12 + [_I] * 6 + [_P, _S, _P]),
    "cd_cross_regression_noalloc_capacity": (_S, []),
    "cd_cross_regression_noalloc": (_I, [_P] * 8 + [_I] * 6 + [_P]),
    "cd_spatial_filter": (_I, [_P] * 9 + [_I] * 4 + [_P]),
    "cd_spatial_filter_grad": (_I, [_P] * 10 + [_I] * 4 + [_P]),
    "cd_spatial_filter_stored": (_I, [_P] * 10 + [_I] * 4 + [_P]),
    "cd_spatial_filter_grad_stored": (_I, [_P] * 6 + [_I] * 3 + [_P]),
    "cd_reproject": (_I, [_P, _I, _P, _P, _P] + [_P] * 8 + [_I] * 3 + [_P]),
    "cd_erode3x3": (_I, [_P, _P, _I, _I, _I, _P]),
    "cd_temporal_screening": (_I, [_P] * 10 + [_I] * 5 + [_P]),
    "cd_erode_temporal_screening": (_I, [_P] * 11 + [_I] * 5 + [_P]),
    "cd_prepare_input": (_I, [_P, _P, _P, _P, _S, _P]),
    "cd_aggregation_workspace_size": (_S, [_I, _I, _I]),
    "cd_aggregation_loss": (_I, [_P] * 22 + [_I] * 3 + [_P, _S, _P]),
    "cd_filter_aggregate_workspace_size": (_S, [_I, _I, _I]),
    "cd_filter_aggregate": (_I, [_P] * 17 + [_I] * 4 + [_P, _S, _P]),
    "cd_unet_param_count": (_S, []),
    "cd_unet_workspace_size": (_S, [_I] * 3),
    "cd_unet_forward": (_I, [_P] * 8 + [_I] * 3 + [_P, _S, _P]),
    "cd_unet_backward": (_I, [_P] * 4 + [_I] * 3 + [_P, _S, _P]),
    "cd_adam_update": (_I, [_P] * 4 + [_I, _P] + [_F] * 4 + [_P]),
    "cd_unet_conv3x3_workspace_size": (_S, [_I, _I]),
    "cd_unet_conv3x3": (_I, [_P] * 4 + [_I] * 6 + [_P, _S, _P]),
    "cd_unet_conv3x3_wgrad_workspace_size": (_S, [_I] * 5),
    "cd_unet_conv3x3_wgrad": (_I, [_P] * 3 + [_I] * 5 + [_P, _S, _P]),
    "cd_fp32_fma_probe": (_I, [_P, _I, _I, _P]),
    "cd_mbar_timeout_probe": (_I, [_P, _I, _I, _P]),
    "cd_image_kernel_error_flags": (_I, []),
    "cd_set_persistent_kernels": (None, [_I]),
    "cd_set_unet_conv_stacked": (None, [_I]),
}

# kernels each entry point launches (for the launch count of bench.py)
KERNELS_PER_CALL = {
    "cd_cross_regression": 3, "cd_cross_regression_fp64_fallback": 3, "cd_cross_regression_grad": 10,
    "cd_cross_regression_keep": 3, "cd_cross_regression_grad_kept": 7, "cd_spatial_filter": 1, "cd_spatial_filter_grad": 1, "cd_spatial_filter_stored": 1, "cd_spatial_filter_grad_stored": 1,
    "cd_reproject": 1,   # 2 for the three 3-channel tensors of the step (ops.reproject passes the count)
    "cd_erode3x3": 1, "cd_temporal_screening": 1, "cd_erode_temporal_screening": 1,
    "cd_prepare_input": 1, "cd_aggregation_loss": 2, "cd_filter_aggregate": 2,
    "cd_unet_forward": 22, "cd_unet_backward": 42, "cd_adam_update": 2, "cd_unet_conv3x3": 2,
    "cd_unet_conv3x3_wgrad": 2,
}
LAUNCHES = {"count": 0}

_lib = None
_lock = threading.Lock()


class CudaOpError(RuntimeError):
    """A CUDA launch or runtime call inside the library failed (CD_ECUDA)."""


def lib() -> ctypes.CDLL:
    """Load libcdops.so once and attach the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is not built; run `python -c 'import __graft_entry__ as g; g.build()'` "
                    "or `make -C cross-denoiser_b200/csrc` first")
            handle = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def check(status: int, op: str, kernels: int | None = None) -> None:
    """Raise the Python analogue of a non-zero cd_status; count launches
    (`kernels` when the entry point's count depends on its arguments)."""
    if status == CD_OK:
        LAUNCHES["count"] += KERNELS_PER_CALL.get("cd_" + op, 0) if kernels is None else kernels
        return
    msg = lib().cd_get_last_error().decode(errors="replace")
    if status == CD_EINVAL:
        raise ValueError(f"{op}: {msg}")
    if status == CD_ENOMEM:
        raise MemoryError(f"{op}: {msg}")
    raise CudaOpError(f"{op}: {msg}")
