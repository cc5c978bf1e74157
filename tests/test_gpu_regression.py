"""CrossRegression on the GPU against the oracle, the golden reference
outputs and the live reference kernel, within rtol 1e-4 (absolute floor 1e-5
for outputs that the reference clamps at zero); variance outputs; batches;
known answers and argument errors."""
import numpy as np
import pytest
import torch

from gpu_util import N, T, frames, needs_reference
from helpers import assert_close, golden, golden_names
from oracle import oracle as orc
from oracle import reference as ref

pytestmark = pytest.mark.gpu
ATOL = 1e-5


def run(cd, y1, y2, alb, nrm, win, sp, rs=1):
    o = cd.ops.cross_regression(T(y1), T(y2), T(alb), T(nrm), win_size=win, sparsity=sp, recon_scale=rs)
    torch.cuda.synchronize()
    return [N(x) for x in o]


def inputs(cd, H, W, seed):
    _, f = frames(cd, H, W, seed=seed)
    return np.log1p(f["color"]), np.log1p(f["color2"]), f["albedo"], f["normal"]


@pytest.mark.parametrize("name", golden_names("regression_"))
def test_golden(cd, cuda, name):
    g = golden(name)
    o = run(cd, g["in_imga"], g["in_imgb"], g["in_albedo"], g["in_normal"], int(g["attr_win_size"]),
            int(g["attr_sparsity"]), int(g["attr_recon_scale"]))
    for x, key in zip(o, ("ref_outa", "ref_outb", "ref_vara", "ref_varb")):
        assert_close(x, g[key], f"{name} {key}", atol=ATOL)


@pytest.mark.parametrize("win,sp,rs", [(11, 4, 1), (15, 4, 1), (17, 4, 1), (19, 4, 1), (15, 4, 2), (17, 4, 4),
                                       (9, 2, 1), (7, 1, 1), (5, 8, 8)])
def test_vs_oracle(cd, cuda, win, sp, rs):
    y1, y2, alb, nrm = inputs(cd, 128, 160, seed=win * 10 + sp)
    o = run(cd, y1, y2, alb, nrm, win, sp, rs)
    r = orc.cross_regression(y1, y2, alb, nrm, win, sp, rs)
    for i, nm in enumerate(("outa", "outb", "vara", "varb")):
        assert_close(o[i], r[i], nm, atol=ATOL)


def unaligned(x):
    """x in a contiguous tensor whose data starts 4 bytes past a 16-byte
    boundary."""
    t = T(x)
    buf = torch.empty(t.numel() + 1, dtype=t.dtype, device=t.device)
    v = buf[1:].view(t.shape)
    v.copy_(t)
    return v


@pytest.mark.parametrize("H,W,win,sp", [(50, 70, 7, 2), (45, 63, 5, 1), (36, 42, 9, 3)])
def test_width_not_multiple_of_4(cd, cuda, H, W, win, sp):
    """Widths with W % 4 != 0 take the per-pixel variance kernel."""
    y1, y2, alb, nrm = inputs(cd, H, W, seed=H + W)
    o = run(cd, y1, y2, alb, nrm, win, sp)
    r = orc.cross_regression(y1, y2, alb, nrm, win, sp, 1)
    for i, nm in enumerate(("outa", "outb", "vara", "varb")):
        assert_close(o[i], r[i], f"{nm} {H}x{W}", atol=ATOL)


def test_unaligned_images(cd, cuda):
    """Images not 16-byte aligned take the per-pixel variance kernel and give
    the same bits as aligned ones."""
    y1, y2, alb, nrm = inputs(cd, 64, 96, seed=4)
    o = cd.ops.cross_regression(unaligned(y1), unaligned(y2), T(alb), T(nrm), win_size=11, sparsity=4)
    torch.cuda.synchronize()
    r = run(cd, y1, y2, alb, nrm, 11, 4)
    for x, y, nm in zip(o, r, ("outa", "outb", "vara", "varb")):
        np.testing.assert_array_equal(N(x), y, err_msg=nm)


def test_batches_are_independent(cd, cuda):
    a = inputs(cd, 64, 96, seed=1)
    b = inputs(cd, 64, 96, seed=2)
    both = [np.concatenate([x, y]) for x, y in zip(a, b)]
    o = run(cd, *both, 15, 4)
    oa = run(cd, *a, 15, 4)
    ob = run(cd, *b, 15, 4)
    for i in range(4):
        np.testing.assert_array_equal(o[i][0:1], oa[i])
        np.testing.assert_array_equal(o[i][1:2], ob[i])


def test_production_size(cd, cuda):
    y1, y2, alb, nrm = inputs(cd, 1080, 1920, seed=9)
    o = run(cd, y1, y2, alb, nrm, 15, 4)
    r = orc.cross_regression(y1, y2, alb, nrm, 15, 4, 1)
    for i, nm in enumerate(("outa", "outb", "vara", "varb")):
        assert_close(o[i], r[i], nm + " 1080p", atol=ATOL)


@needs_reference
@pytest.mark.parametrize("win", [11, 15, 17, 19])
def test_vs_reference_kernel(cd, cuda, win):
    y1, y2, alb, nrm = inputs(cd, 256, 320, seed=win)
    o = run(cd, y1, y2, alb, nrm, win, 4)
    r = ref.cross_regression(T(y1), T(y2), T(alb), T(nrm), win, 4, 1)
    torch.cuda.synchronize()
    for i, nm in enumerate(("outa", "outb", "vara", "varb")):
        assert_close(o[i], N(r[i]), nm + " vs reference", atol=ATOL)


def test_constant_target(cd, cuda):
    H, W = 64, 64
    c = np.full((1, H, W, 3), 0.7, np.float32)
    rng = np.random.default_rng(0)
    alb = rng.uniform(0.1, 0.9, (1, H, W, 3)).astype(np.float32)
    o = run(cd, c, c, alb, alb, 15, 4)
    assert_close(o[0], np.full_like(o[0], 0.7), "constant", rtol=1e-4)


def test_argument_errors(cd, cuda):
    x = torch.zeros((1, 64, 64, 3), device=cuda)
    with pytest.raises(ValueError, match="recon_scale"):
        cd.ops.cross_regression(x, x, x, x, win_size=15, sparsity=2, recon_scale=4)
    with pytest.raises(ValueError, match="divisible"):
        cd.ops.cross_regression(x[:, :62], x[:, :62], x[:, :62], x[:, :62], win_size=15, sparsity=4)
    with pytest.raises(ValueError):
        cd.ops.cross_regression(x[:, :8, :8], x[:, :8, :8], x[:, :8, :8], x[:, :8, :8], win_size=17, sparsity=4)


def test_fp64_fallback(cd, cuda):
    """cd_cross_regression_fp64_fallback: with an unreachable limit nothing
    falls back and the outputs are the reference path's bit for bit; with a
    limit of 1 every (centre, channel, buffer) is re-solved in double, and
    the outputs stay within the op tolerance of the FP64 restatement."""
    from oracle import regression_fp64 as r64
    y1, y2, alb, nrm = inputs(cd, 32, 48, seed=5)
    win, sp = 9, 4
    base = run(cd, y1, y2, alb, nrm, win, sp)
    cnt = torch.zeros((1,), dtype=torch.int32, device="cuda:0")
    o = cd.ops.cross_regression(T(y1), T(y2), T(alb), T(nrm), win_size=win, sparsity=sp, fp64_cond_limit=1e30,
                                fallback_count=cnt)
    torch.cuda.synchronize()
    assert int(cnt.item()) == 0
    for a, b in zip(o, base):
        np.testing.assert_array_equal(N(a), b)
    cnt.zero_()
    o = cd.ops.cross_regression(T(y1), T(y2), T(alb), T(nrm), win_size=win, sparsity=sp, fp64_cond_limit=1.0,
                                fallback_count=cnt)
    torch.cuda.synchronize()
    assert int(cnt.item()) == (32 // sp) * (48 // sp) * 3 * 2
    ref = r64.cross_regression(*[torch.from_numpy(a).double() for a in (y1, y2, alb, nrm)], win, sp, 1)
    for a, b, nm in zip(o, ref, ("outa", "outb", "vara", "varb")):
        assert_close(N(a), b.numpy().astype(np.float32), f"fp64 fallback {nm}", atol=ATOL)
    with pytest.raises(ValueError):
        cd.ops._lib.check(cd.ops._lib.lib().cd_cross_regression_fp64_fallback(
            *[None] * 8, 1, 32, 48, win, sp, 1, 0.0, None, None, 0, None), "cross_regression_fp64_fallback")
