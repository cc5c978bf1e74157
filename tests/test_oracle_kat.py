"""Known-answer tests of the CPU oracle, derived from the reference formulas
by hand (no GPU)."""
import numpy as np
import pytest

from helpers import assert_close, assert_equal
from oracle import oracle as orc

rng = np.random.default_rng(0)


def _img(H, W, C=3, lo=0.0, hi=1.0):
    return rng.uniform(lo, hi, (1, H, W, C)).astype(np.float32)


def test_regression_constant_image():
    """A constant target is reproduced up to the 1e-3 ridge
    (ops/regression.cu.cc:458-461) and has zero variance."""
    H, W = 32, 48
    c = np.full((1, H, W, 3), 0.7, np.float32)
    oa, ob, va, vb = orc.cross_regression(c, c, _img(H, W), _img(H, W, lo=-1), 15, 4, 1)
    assert_close(oa, np.full_like(oa, 0.7), "outa", rtol=1e-4)
    assert_close(ob, np.full_like(ob, 0.7), "outb", rtol=1e-4)
    assert va.max() < 1e-12 and vb.max() < 1e-12


def test_regression_linear_in_albedo():
    """A target that is an affine function of the albedo is fitted exactly
    (the albedo difference is a regression feature)."""
    H, W = 32, 32
    alb = _img(H, W, lo=0.1, hi=0.9)
    y = (0.3 + 2.0 * alb).astype(np.float32)
    f = _img(H, W)
    oa, *_ = orc.cross_regression(f, y, alb, np.zeros_like(alb), 11, 4, 1)
    # outa predicts imgb (= y) from imga's features
    assert_close(oa, y, "outa", rtol=2e-3, atol=1e-4)


def test_variance_known_answer():
    img = np.zeros((1, 3, 3, 3), np.float32)
    img[0, 1, 1] = [3.0, 0.0, 0.0]
    v = orc.variance(img)
    # centre: neighbours all 0 -> |0 - 3|^2 = 9; corner (0,0): neighbours
    # (0,1),(1,0),(1,1) -> mean x = 1 -> 1
    assert v[0, 1, 1, 0] == 9.0
    assert v[0, 0, 0, 0] == 1.0


def test_spatial_filter_zero_band_is_box_sum():
    H, W, win = 16, 20, 5
    a, b = _img(H, W), _img(H, W)
    acca, accb, wa, wb = orc.spatial_filter(a, b, _img(H, W), _img(H, W), np.zeros((1, H, W, 5), np.float32), win)
    assert np.all(wa == 25.0) and np.all(wb == 25.0)
    # interior pixel: plain 5x5 sum
    assert_close(acca[0, 8, 10], a[0, 6:11, 8:13].reshape(-1, 3).sum(0), "box sum", rtol=1e-5)


def test_spatial_filter_grad_zero_upstream():
    H, W = 12, 12
    args = [_img(H, W) for _ in range(4)] + [_img(H, W, 5)]
    o = orc.spatial_filter(*args, 5, partials=True)
    z3, z1 = np.zeros((1, H, W, 3), np.float32), np.zeros((1, H, W, 1), np.float32)
    g = orc.spatial_filter_grad_from_partials(z3, z3, z1, z1, o[4], o[5])
    assert np.all(g == 0)
    # d wsum_A / d band_4 = -sum_t w_t d(p,t): negative unless only the centre tap
    g = orc.spatial_filter_grad_from_partials(z3, z3, z1 + 1, z1, o[4], o[5])
    assert np.all(g[..., 4] < 0) and np.all(g[..., 1] == 0)


def _gbuf(H, W):
    z = np.full((1, H, W, 1), 10.0, np.float32)
    lin = np.concatenate([z, np.full_like(z, 0.5), np.zeros_like(z)], -1)
    n = np.broadcast_to(np.array([0, 0.6, 0.8], np.float32), (1, H, W, 3)).copy()
    return lin, n


def test_reproject_identity():
    """mvec = 0 with identical G-buffers: every pixel but the 1-px top/left
    border (rounded position < 1, ops/reproject.cu.cc:38) reprojects onto
    itself."""
    H, W = 24, 32
    lin, n = _gbuf(H, W)
    x = _img(H, W)
    one = np.ones((1, H, W, 1), np.float32)
    s, (o,) = orc.reproject(np.zeros((1, H, W, 3), np.float32), [x], lin, lin, n, n, np.zeros_like(n), one, one)
    assert not s[0, 0, :, 0].any() and not s[0, :, 0, 0].any()
    assert s[0, 1:, 1:, 0].all()
    assert_equal(o[0, 1:, 1:], x[0, 1:, 1:], "identity")
    assert np.all(o[0, 0] == 0)


def test_reproject_integer_shift():
    H, W = 24, 32
    lin, n = _gbuf(H, W)
    x = _img(H, W, 2)
    one = np.ones((1, H, W, 1), np.float32)
    mv = np.zeros((1, H, W, 3), np.float32)
    mv[..., 0] = 2.0 / W                      # previous position = pos + (2, 0)
    s, (o,) = orc.reproject(mv, [x], lin, lin, n, n, np.zeros_like(n), one, one)
    assert s[0, 1:, 1:W - 3, 0].all()
    assert_close(o[0, 1:, 1:W - 3], x[0, 1:, 3:W - 1], "shift", rtol=1e-6)


def test_reproject_rejections():
    H, W = 16, 16
    lin, n = _gbuf(H, W)
    x = _img(H, W)
    one = np.ones((1, H, W, 1), np.float32)
    mv = np.zeros((1, H, W, 3), np.float32)
    # opacity 0 -> rejected, outputs zero
    s, (o,) = orc.reproject(mv, [x], lin, lin, n, n, np.zeros_like(n), np.zeros_like(one), one)
    assert not s.any() and np.all(o == 0)
    # depth jump beyond 10 * (fwidth + 0.01) -> rejected
    lin2 = lin.copy()
    lin2[..., 0] += 10.0
    s, _ = orc.reproject(mv, [x], lin, lin2, n, n, np.zeros_like(n), one, one)
    assert not s.any()
    # normal flip with small fwidth -> rejected
    s, _ = orc.reproject(mv, [x], lin, lin, n, -n, np.zeros_like(n), one, one)
    assert not s.any()
    # far out of the screen -> rejected
    mv[..., 0] = 5.0
    s, _ = orc.reproject(mv, [x], lin, lin, n, n, np.zeros_like(n), one, one)
    assert not s.any()


def test_reproject_fallback_box():
    """When no bilinear tap is valid the 3x3 box around the rounded position
    is averaged (ops/reproject.cu.cc:179-225)."""
    H, W = 16, 16
    lin, n = _gbuf(H, W)
    x = _img(H, W, 1)
    one = np.ones((1, H, W, 1), np.float32)
    popac = one.copy()
    popac[0, 8, 8] = 0.0                        # the only bilinear tap of pixel (8, 8)
    mv = np.zeros((1, H, W, 3), np.float32)
    s, (o,) = orc.reproject(mv, [x], lin, lin, n, n, np.zeros_like(n), one, popac)
    assert s[0, 8, 8, 0]
    box = [x[0, 7 + k // 3, 7 + k % 3, 0] for k in range(9) if k != 4]
    assert_close(o[0, 8, 8, 0], np.float32(np.sum(np.float32(box), dtype=np.float32) / 8), "box", rtol=1e-6)


def test_erosion():
    m = np.ones((1, 5, 6, 1), np.uint8)
    m[0, 2, 3] = 0
    e = orc.erode3x3(m)
    assert e[0, 1:4, 2:5].max() == 0 and e.sum() == 30 - 9


def test_temporal_rules():
    H, W = 12, 14
    a, b = _img(H, W), _img(H, W)
    cur = (a + b) * np.float32(0.5)
    ones = np.ones((1, H, W, 1), np.float32)
    # eroded mask below 1 -> current values, success 0
    o, o1, o2, s = orc.temporal_screening(a, b, cur + 5, a + 5, b + 5, ones * 0.5, 7, 1)
    assert_equal(o, cur, "current"), assert_equal(o1, a, "c1")
    assert not s.any()
    # history equal to the current frame: accepted exactly where the pixel is
    # strictly inside its 7x7 window's range in every channel
    o, o1, o2, s = orc.temporal_screening(a, b, cur, a, b, ones, 7, 1)
    expect = np.zeros((H, W), bool)
    for y in range(H):
        for x in range(W):
            win = cur[0, max(0, y - 3):y + 4, max(0, x - 3):x + 4].reshape(-1, 3)
            v = cur[0, y, x]
            expect[y, x] = np.all(win.min(0) < v) and np.all(v < win.max(0))
    assert_equal(s[0, ..., 0].astype(bool), expect, "accept rule")
    # constant frame: min == max, strict overlap fails everywhere
    c = np.full_like(a, 0.25)
    *_, s = orc.temporal_screening(c, c, c, c, c, ones, 7, 1)
    assert not s.any()
