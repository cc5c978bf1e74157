"""B200 (sm_100a) per-frame hot path of the online cross-regression denoiser.

A drop-in for the reference's TensorFlow custom ops (scripts/ops.py): the
op functions in :mod:`.ops` keep the reference names, argument order,
attributes and NHWC layouts, and run hand-written CUDA kernels through the C
ABI of include/cd_ops.h (libcdops.so, built in-tree).

The directory name is not a Python identifier; the package is registered as
``cross_denoiser_b200`` by ``__graft_entry__.load_package()`` (the tests,
bench.py and smoke() do this), or by any importlib loader pointed at this
directory.
"""
from . import _lib, frames, ops, replicas, serve, step, synth, unet  # noqa: F401
from .ops import (Reproject, cross_regression, erode3x3, erode_temporal_screening,  # noqa: F401
                  reproject, spatial_filter, spatial_filter_grad, temporal_screening)

__version__ = "0.1.0"
