"""The C ABI library without a GPU: it loads, exports every entry point that
include/cd_ops.h declares, and rejects invalid arguments before touching the
device.  The op surface refuses CPU tensors (there is no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "cd_ops.h")).read()
    return sorted(set(re.findall(r"^CD_API\s+[\w\s\*]+?\b(cd_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol(cd):
    lib = cd._lib.lib()
    names = header_functions()
    assert len(names) >= 9
    for n in names:
        assert hasattr(lib, n), f"libcdops.so does not export {n}"
    assert set(names) <= set(cd._lib.SIGNATURES), "ctypes signatures missing for some entry points"
    assert lib.cd_abi_version() == 1


def test_invalid_arguments_are_rejected_without_a_device(cd):
    lib = cd._lib.lib()
    p = ctypes.c_void_p(16)          # never dereferenced: validation fails first
    st = ctypes.c_void_p(0)
    # recon_scale > sparsity (ops/regression.cc:134-135)
    rc = lib.cd_cross_regression(*([p] * 8), 1, 64, 64, 15, 2, 4, p, 1 << 20, st)
    assert rc == cd._lib.CD_EINVAL
    assert b"recon_scale" in lib.cd_get_last_error()
    # H not divisible by recon_scale (ops/regression.cc:159-160)
    rc = lib.cd_cross_regression(*([p] * 8), 1, 66, 64, 15, 4, 4, p, 1 << 20, st)
    assert rc == cd._lib.CD_EINVAL and b"divisible" in lib.cd_get_last_error()
    # window radius not smaller than the image (the reference reads out of bounds)
    rc = lib.cd_cross_regression(*([p] * 8), 1, 8, 8, 17, 4, 1, p, 1 << 20, st)
    assert rc == cd._lib.CD_EINVAL
    # workspace too small
    rc = lib.cd_cross_regression(*([p] * 8), 1, 64, 64, 15, 4, 1, p, 16, st)
    assert rc == cd._lib.CD_ENOMEM
    # null pointers
    rc = lib.cd_spatial_filter(*([None] * 9), 1, 8, 8, 5, st)
    assert rc == cd._lib.CD_EINVAL
    rc = lib.cd_temporal_screening(*([p] * 10), 1, 8, 8, 0, 1, st)
    assert rc == cd._lib.CD_EINVAL
    arr = (ctypes.c_void_p * 9)(*([16] * 9))
    ch = (ctypes.c_int * 9)(*([3] * 9))
    rc = lib.cd_reproject(p, 9, arr, ch, arr, *([p] * 8), 1, 8, 8, st)
    assert rc == cd._lib.CD_EINVAL
    rc = lib.cd_erode3x3(None, p, 1, 8, 8, st)
    assert rc == cd._lib.CD_EINVAL
    assert lib.cd_cross_regression_workspace_size(2, 64, 32, 4) == (2 * 2 * 16 * 8 * 18 + 2 * 2 * 64 * 32) * 4


def test_noalloc_checks_arguments_before_capacity(cd):
    """The entry point without a workspace reports invalid arguments as the
    regular entry point does (CD_EINVAL), even for a frame too large for its
    built-in array; a valid oversized frame is CD_ENOMEM.  Neither touches
    the device."""
    lib = cd._lib.lib()
    p = ctypes.c_void_p(16)
    st = ctypes.c_void_p(0)
    H, W = 2160, 3840
    assert lib.cd_cross_regression_workspace_size(1, H, W, 4) > lib.cd_cross_regression_noalloc_capacity()
    rc = lib.cd_cross_regression_noalloc(*([p] * 8), 1, H, W, 15, 2, 4, st)     # recon_scale > sparsity
    assert rc == cd._lib.CD_EINVAL and b"recon_scale" in lib.cd_get_last_error()
    rc = lib.cd_cross_regression_noalloc(*([p] * 7), None, 1, H, W, 15, 4, 1, st)
    assert rc == cd._lib.CD_EINVAL and b"null" in lib.cd_get_last_error()
    rc = lib.cd_cross_regression_noalloc(*([p] * 8), 1, H, W, 15, 4, 1, st)
    assert rc == cd._lib.CD_ENOMEM and b"built-in array" in lib.cd_get_last_error()


def test_ops_refuse_cpu_tensors(cd):
    x = torch.zeros((1, 8, 8, 3))
    with pytest.raises(ValueError, match="CUDA"):
        cd.ops.cross_regression(x, x, x, x, win_size=3, sparsity=2)
    with pytest.raises(ValueError, match="CUDA"):
        cd.ops.spatial_filter(x, x, x, x, torch.zeros((1, 8, 8, 5)), win_size=3)
    with pytest.raises(ValueError, match="CUDA"):
        cd.ops.Reproject(x, [x], x, x, x, x, x, x[..., :1], x[..., :1])
    with pytest.raises(ValueError, match="CUDA"):
        cd.ops.temporal_screening(x, x, x, x, x, x[..., :1], 7, 1)


def test_python_error_mapping(cd):
    with pytest.raises(ValueError, match="recon_scale"):
        cd._lib.check(cd._lib.lib().cd_cross_regression(*([ctypes.c_void_p(16)] * 8), 1, 64, 64, 15, 2, 4,
                                                          ctypes.c_void_p(16), 1 << 20, ctypes.c_void_p(0)),
                      "cross_regression")
