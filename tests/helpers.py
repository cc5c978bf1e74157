"""Comparison helpers and tolerances shared by the tests.

Tolerances (per value, |a - b| <= atol + rtol * |b|):
  * masks and temporal-screening outputs: bit-exact;
  * floating-point outputs: rtol = 1e-4 (the parity bar for FP32 outputs and
    gradients), with a small absolute floor for values that round to ~0
    (clamped regression outputs, cancelling gradient sums) stated per test.
"""
from __future__ import annotations

import os

import numpy as np

RTOL = 1e-4
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def assert_close(a, b, what, rtol=RTOL, atol=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, f"{what}: shape {a.shape} != {b.shape}"
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin), f"{what}: non-finite pattern differs"
    diff = np.abs(a[fin] - b[fin])
    bad = diff > atol + rtol * np.abs(b[fin])
    if bad.any():
        rel = diff / np.maximum(np.abs(b[fin]), 1e-30)
        raise AssertionError(
            f"{what}: {int(bad.sum())}/{bad.size} values outside atol={atol:g} rtol={rtol:g}; "
            f"max |diff| {diff.max():.3g}, max rel {rel[bad].max():.3g}")


def assert_equal(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} != {b.shape}"
    ne = a != b
    if a.dtype.kind == "f":
        ne &= ~(np.isnan(a) & np.isnan(b))
    assert not ne.any(), f"{what}: {int(ne.sum())}/{ne.size} values differ"


def golden(name):
    path = os.path.join(GOLDEN, name + ".npz")
    return dict(np.load(path))


def golden_names(prefix):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.startswith(prefix) and f.endswith(".npz"))
