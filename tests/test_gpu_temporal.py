"""Erosion and temporal screening on the GPU: bit-exact against the oracle,
the golden reference outputs and the live reference kernel; the fused
erosion + screening kernel equals the two-op sequence."""
import numpy as np
import pytest
import torch

from gpu_util import N, T, frames, needs_reference
from helpers import assert_equal, golden, golden_names
from oracle import oracle as orc
from oracle import reference as ref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names("temporal_"))
def test_golden(cd, cuda, name):
    g = golden(name)
    wc, wp = int(g["attr_win_curr"]), int(g["attr_win_prev"])
    ins = [T(g[k]) for k in ("in_current1", "in_current2", "in_prev", "in_prev1", "in_prev2")]
    ero = cd.ops.erode3x3(T(g["in_reproj_mask"]))
    assert_equal(N(ero), g["in_reproj_success"], "erosion")
    o = cd.ops.temporal_screening(*ins, T(g["in_reproj_success"]), wc, wp)
    f = cd.ops.erode_temporal_screening(*ins, T(g["in_reproj_mask"]), wc, wp)
    torch.cuda.synchronize()
    for i, key in enumerate(("ref_output", "ref_output1", "ref_output2", "ref_success")):
        assert_equal(N(o[i]), g[key], f"{name} {key}")
        assert_equal(N(f[i]), g[key], f"{name} fused {key}")
    assert_equal(N(f[4]), g["in_reproj_success"], "fused eroded mask")


def inputs(cd, H, W, B, seed):
    rng = np.random.default_rng(seed)
    f0, f1 = frames(cd, H, W, seed=seed)
    c1 = np.concatenate([np.log1p(f1["color"])] * B)
    c2 = np.concatenate([np.log1p(f1["color2"])] * B)
    c2[1:] *= 1.1 if B > 1 else 1.0
    prev = (c1 + c2) * np.float32(0.5) + rng.normal(0, 0.1, c1.shape).astype(np.float32)
    p1 = c1 + rng.normal(0, 0.2, c1.shape).astype(np.float32)
    p2 = c2 + rng.normal(0, 0.2, c1.shape).astype(np.float32)
    mask = rng.uniform(size=(B, H, W, 1)) > 0.03
    return c1, c2, prev, p1, p2, mask


@pytest.mark.parametrize("H,W,B,wc,wp", [(96, 128, 2, 7, 1), (61, 77, 1, 5, 3), (40, 40, 1, 1, 1),
                                         (50, 70, 1, 9, 5), (1080, 1920, 1, 7, 1)])
def test_vs_oracle(cd, cuda, H, W, B, wc, wp):
    c1, c2, prev, p1, p2, mask = inputs(cd, H, W, B, seed=H)
    ero = orc.erode3x3(mask)
    ro = orc.temporal_screening(c1, c2, prev, p1, p2, ero, wc, wp)
    ins = [T(x) for x in (c1, c2, prev, p1, p2)]
    me = cd.ops.erode3x3(T(mask))
    o = cd.ops.temporal_screening(*ins, me, wc, wp)
    f = cd.ops.erode_temporal_screening(*ins, T(mask), wc, wp)
    torch.cuda.synchronize()
    assert_equal(N(me), ero, "erosion")
    if wc > 1:
        assert 0.3 < ro[3].mean() < 1.0     # a 1x1 window can never pass the strict overlap test
    for i in range(4):
        assert_equal(N(o[i]), ro[i], f"out{i}")
        assert_equal(N(f[i]), ro[i], f"fused out{i}")


@pytest.mark.parametrize("H,W,B,wc", [(37, 48, 3, 7), (8, 16, 1, 7), (5, 16, 2, 5), (70, 176, 1, 3),
                                       (130, 272, 2, 7), (19, 80, 1, 5)])
def test_persistent_tma_kernel(cd, cuda, H, W, B, wc):
    """Rows a multiple of 16 bytes and win_prev = 1: the fused op takes the
    persistent kernel with TMA-staged tiles (partial tiles at the right and
    bottom edges, boxes reaching past the image, several images, more tiles
    than CTAs and fewer).  Bit-exact against the oracle, the two-op
    sequence and the tile-per-CTA fused kernel; no staging wait ran out."""
    c1, c2, prev, p1, p2, mask = inputs(cd, H, W, B, seed=H + W)
    ero = orc.erode3x3(mask)
    ro = orc.temporal_screening(c1, c2, prev, p1, p2, ero, wc, 1)
    ins = [T(x) for x in (c1, c2, prev, p1, p2)]
    o = cd.ops.temporal_screening(*ins, cd.ops.erode3x3(T(mask)), wc, 1)
    f = cd.ops.erode_temporal_screening(*ins, T(mask), wc, 1)
    torch.cuda.synchronize()
    L = cd._lib.lib()
    try:
        L.cd_set_persistent_kernels(0)
        t = cd.ops.erode_temporal_screening(*ins, T(mask), wc, 1)
        torch.cuda.synchronize()
    finally:
        L.cd_set_persistent_kernels(1)
    assert_equal(N(f[4]), ero, "fused eroded mask")
    for i in range(5):
        assert_equal(N(f[i]), N(t[i]), f"fused out{i} vs the tile-per-CTA kernel")
    for i in range(4):
        assert_equal(N(f[i]), ro[i], f"fused out{i} vs oracle")
        assert_equal(N(f[i]), N(o[i]), f"fused out{i} vs two-op sequence")
    assert L.cd_image_kernel_error_flags() == 0


def test_all_rejected_and_all_accepted(cd, cuda):
    c1, c2, prev, p1, p2, mask = inputs(cd, 32, 32, 1, seed=3)
    ins = [T(x) for x in (c1, c2, prev, p1, p2)]
    o = cd.ops.temporal_screening(*ins, torch.zeros((1, 32, 32, 1), device=cuda), 7, 1)
    assert not N(o[3]).any()
    assert_equal(N(o[0]), (c1 + c2) * np.float32(0.5), "current")
    cur = (c1 + c2) * np.float32(0.5)
    same = [T(x) for x in (c1, c2, cur, c1, c2)]
    o = cd.ops.temporal_screening(*same, torch.ones((1, 32, 32, 1), device=cuda), 7, 1)
    ro = orc.temporal_screening(c1, c2, cur, c1, c2, np.ones((1, 32, 32, 1), np.float32), 7, 1)
    assert_equal(N(o[3]), ro[3], "history == current")


@needs_reference
def test_vs_reference_kernel(cd, cuda):
    c1, c2, prev, p1, p2, mask = inputs(cd, 256, 384, 1, seed=5)
    ins = [T(x) for x in (c1, c2, prev, p1, p2)]
    ero = ref.erode3x3(T(mask))
    r = ref.temporal_screening(*ins, ero, 7, 1)
    f = cd.ops.erode_temporal_screening(*ins, T(mask), 7, 1)
    torch.cuda.synchronize()
    for i in range(4):
        assert_equal(N(f[i]), N(r[i]), f"out{i} vs reference")


def test_argument_errors(cd, cuda):
    x = torch.zeros((1, 8, 8, 3), device=cuda)
    m = torch.zeros((1, 8, 8, 1), device=cuda)
    with pytest.raises(ValueError):
        cd.ops.temporal_screening(x, x, x, x, x, m, 0, 1)
    with pytest.raises(ValueError):
        cd.ops.temporal_screening(x, x, x, x, x[:, :4], m, 7, 1)
    with pytest.raises(ValueError):
        cd.ops.erode3x3(m)            # needs a bool mask
