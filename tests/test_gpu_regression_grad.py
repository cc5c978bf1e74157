"""CrossRegression backward (cd_cross_regression_grad) against torch.autograd
through the float64 restatement oracle/regression_fp64.py.

The reference has no gradient for this op, so the FP64 restatement of its
forward (itself checked against central differences in
test_oracle_regression_fp64.py) is the oracle.  FP32 gradient vs FP64
gradient tolerance, per element of each output tensor:
    |g - g64| <= 1e-4 * |g64| + 1e-4 * max|g64|
i.e. rtol 1e-4 with an absolute floor of 1e-4 of the tensor's largest
magnitude (entries that are sums of many terms of both signs end near zero,
where a relative bound alone is meaningless; the forward alone differs from
FP64 by up to ~7e-5 relative, and the backward passes through two 6x6
solves and the reconstruction's quotient).
"""
import numpy as np
import pytest
import torch

from gpu_util import T, N, frames
from oracle import regression_fp64 as r64

pytestmark = pytest.mark.gpu
FLOOR_OF_MAX, RTOL_EL = 1e-4, 1e-4
NAMES = ("grad_imga", "grad_imgb", "grad_albedo", "grad_normal")


def inputs(cd, H, W, seed, B=1):
    out = []
    for b in range(B):
        _, f = frames(cd, H, W, seed=seed + b)
        out.append((np.log1p(f["color"]), np.log1p(f["color2"]), f["albedo"], f["normal"]))
    return [np.concatenate([o[i] for o in out]) for i in range(4)]


def upstream(B, H, W, rs, seed, with_var=True):
    g = np.random.default_rng(seed)
    go = [g.standard_normal((B, H // rs, W // rs, 3)).astype(np.float32) for _ in range(2)]
    gv = [g.standard_normal((B, H, W, 1)).astype(np.float32) if with_var else None for _ in range(2)]
    return go + gv


def fp64_grads(ins, ups, win, sp, rs):
    x = [torch.from_numpy(a).double().requires_grad_(True) for a in ins]
    outs = r64.cross_regression(*x, win, sp, rs)
    loss = 0
    for o, g in zip(outs, ups):
        if g is not None:
            loss = loss + (o * torch.from_numpy(g).double()).sum()
    loss.backward()
    return [t.grad.numpy() for t in x]


def check(got, want, what):
    for g, w, nm in zip(got, want, NAMES):
        err = np.abs(g.astype(np.float64) - w)
        bound = FLOOR_OF_MAX * np.abs(w).max() + RTOL_EL * np.abs(w)
        bad = err > bound
        assert not bad.any(), (f"{what} {nm}: {bad.sum()} of {bad.size} beyond tolerance, "
                               f"max err {err.max():.3g}, max|g64| {np.abs(w).max():.3g}")


# The last two cases reach the backward's unstaged forms: at sparsity 1 and
# window 9 the staged pixel- and tap-side records exceed shared memory; at
# window 63 a centre has more than 64 candidate columns, so the centre-side
# pass runs one thread per centre testing the range rule in its loop.
@pytest.mark.parametrize("H,W,win,sp,rs", [(16, 20, 5, 1, 1), (24, 32, 7, 2, 1), (24, 32, 7, 2, 2),
                                            (32, 40, 9, 4, 1), (32, 40, 11, 4, 2), (24, 32, 5, 4, 4),
                                            (24, 32, 9, 1, 1), (72, 80, 63, 4, 1)])
def test_vs_fp64_autograd(cd, cuda, H, W, win, sp, rs):
    ins = inputs(cd, H, W, seed=H + win)
    ups = upstream(1, H, W, rs, seed=win * 7 + sp)
    got = cd.ops.cross_regression_grad(*[T(u) if u is not None else None for u in ups],
                                       *[T(a) for a in ins], win, sp, rs)
    torch.cuda.synchronize()
    check([N(g) for g in got], fp64_grads(ins, ups, win, sp, rs), f"{H}x{W} win {win} sp {sp} rs {rs}")


def test_outputs_only(cd, cuda):
    """NULL variance gradients: the variances reach the loss only through
    the regression and the reconstruction."""
    H, W, win, sp, rs = 24, 32, 7, 2, 1
    ins = inputs(cd, H, W, seed=3)
    ups = upstream(1, H, W, rs, seed=4, with_var=False)
    got = cd.ops.cross_regression_grad(T(ups[0]), T(ups[1]), None, None, *[T(a) for a in ins], win, sp, rs)
    check([N(g) for g in got], fp64_grads(ins, ups, win, sp, rs), "no variance gradients")


def test_batch(cd, cuda):
    H, W, win, sp, rs = 16, 24, 5, 2, 1
    ins = inputs(cd, H, W, seed=11, B=2)
    ups = upstream(2, H, W, rs, seed=12)
    got = cd.ops.cross_regression_grad(*[T(u) for u in ups], *[T(a) for a in ins], win, sp, rs)
    check([N(g) for g in got], fp64_grads(ins, ups, win, sp, rs), "batch of 2")


def test_autograd_function(cd, cuda):
    """cross_regression is differentiable through torch.autograd when an
    input requires grad, and the gradient is cd_cross_regression_grad's."""
    H, W, win, sp = 16, 20, 5, 2
    ins = inputs(cd, H, W, seed=21)
    x = [T(a).requires_grad_(True) for a in ins]
    outa, outb, va, vb = cd.ops.cross_regression(*x, win_size=win, sparsity=sp)
    ups = upstream(1, H, W, 1, seed=22)
    loss = sum((o * T(g)).sum() for o, g in zip((outa, outb, va, vb), ups))
    loss.backward()
    direct = cd.ops.cross_regression_grad(*[T(u) for u in ups], *[T(a) for a in ins], win, sp, 1)
    for t, d in zip(x, direct):
        np.testing.assert_array_equal(N(t.grad), N(d))
    # without requires_grad the plain forward runs (no graph)
    o = cd.ops.cross_regression(*[T(a) for a in ins], win_size=win, sparsity=sp)
    assert o[0].grad_fn is None
    np.testing.assert_array_equal(N(o[0]), N(outa.detach()))


@pytest.mark.parametrize("sp,rs", [(4, 1), (2, 2)])
def test_keep_and_kept_are_bit_identical(cd, cuda, sp, rs):
    """cross_regression_keep gives cross_regression's outputs and
    cross_regression_grad_kept cross_regression_grad's, bit for bit (the
    same kernels on the same inputs, the backward without its recompute);
    the autograd path uses the pair."""
    B, H, W, win = 2, 48, 56, 9
    ins = [T(a) for a in inputs(cd, H, W, seed=91, B=B)]
    ups = [None if u is None else T(u) for u in upstream(B, H, W, rs, seed=92)]
    plain = cd.ops.cross_regression(*ins, win_size=win, sparsity=sp, recon_scale=rs)
    kept_outs, ws = cd.ops.cross_regression_keep(*ins, win, sp, rs)
    for a, b in zip(plain, kept_outs):
        assert torch.equal(a, b)
    g_re = cd.ops.cross_regression_grad(*ups, *ins, win, sp, rs)
    g_kept = cd.ops.cross_regression_grad_kept(*ups, *ins, win, sp, rs, ws)
    for a, b, nm in zip(g_re, g_kept, NAMES):
        assert torch.equal(a, b), nm
    x = [t.clone().requires_grad_(True) for t in ins]
    outs = cd.ops.cross_regression(*x, win_size=win, sparsity=sp, recon_scale=rs)
    loss = sum((o * u).sum() for o, u in zip(outs, ups) if u is not None)
    loss.backward()
    for t, b, nm in zip(x, g_re, NAMES):
        assert torch.equal(t.grad, b), f"autograd {nm}"


def test_argument_errors(cd, cuda):
    ins = [T(a) for a in inputs(cd, 16, 20, seed=1)]
    g = torch.zeros((1, 16, 20, 3), device="cuda:0")
    with pytest.raises(ValueError):
        cd.ops.cross_regression_grad(g[:, :8], g, None, None, *ins, 5, 2, 1)
    with pytest.raises(ValueError, match="recon_scale"):
        cd.ops.cross_regression_grad(g, g, None, None, *ins, 5, 2, 4)
    with pytest.raises(ValueError, match="sparsity"):
        cd.ops.cross_regression_grad(g, g, None, None, *ins, 5, 3, 1)
