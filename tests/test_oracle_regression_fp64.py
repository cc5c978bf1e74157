"""The float64 CrossRegression restatement (oracle/regression_fp64.py), which
is the oracle for the regression's backward: its forward against the FP32
C oracle, and its autograd gradient against central finite differences."""
import numpy as np
import torch

from oracle import oracle as orc
from oracle import regression_fp64 as r64


def frame(cd, H, W, seed):
    f = cd.synth.make_sequence(H, W, seed=seed).frame(2)
    return (np.log1p(f["color"].numpy()), np.log1p(f["color2"].numpy()), f["albedo"].numpy(),
            f["normal"].numpy())


def test_forward_matches_fp32_oracle(cd):
    for H, W, win, sp, rs in ((24, 32, 9, 4, 1), (20, 28, 7, 2, 2), (20, 28, 5, 4, 4)):
        ins = frame(cd, H, W, seed=H + win)
        want = orc.cross_regression(*ins, win, sp, rs)
        got = r64.cross_regression(*[torch.from_numpy(a).double() for a in ins], win, sp, rs)
        for a, b, nm in zip(want, got, ("outa", "outb", "vara", "varb")):
            b = b.numpy()
            rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-3)
            assert rel.max() < 2e-4, f"{H}x{W} win {win} sp {sp} rs {rs} {nm}: max rel {rel.max():.3g}"


def test_autograd_matches_central_differences(cd):
    H, W, win, sp, rs = 16, 20, 5, 4, 1
    ins = [torch.from_numpy(a).double().requires_grad_(True) for a in frame(cd, H, W, seed=5)]
    g = torch.Generator().manual_seed(0)
    ws = [torch.randn(s, generator=g, dtype=torch.float64)
          for s in ((1, H, W, 3), (1, H, W, 3), (1, H, W, 1), (1, H, W, 1))]

    def loss(*xs):
        return sum((o * w).sum() for o, w in zip(r64.cross_regression(*xs, win, sp, rs), ws))

    grads = torch.autograd.grad(loss(*ins), ins)
    rng = np.random.default_rng(1)
    h = 1e-6
    for _ in range(24):
        i, y, x, c = rng.integers(4), rng.integers(H), rng.integers(W), rng.integers(3)
        xp = [t.detach().clone() for t in ins]
        xm = [t.detach().clone() for t in ins]
        xp[i][0, y, x, c] += h
        xm[i][0, y, x, c] -= h
        fd = (loss(*xp) - loss(*xm)).item() / (2 * h)
        an = grads[i][0, y, x, c].item()
        assert abs(fd - an) <= 1e-5 * max(abs(fd), 1e-3), (i, y, x, c, fd, an)


def test_idivup_c_semantics():
    # C's truncating division: iDivUp(-3, 4) = 0 + 1 = 1, iDivUp(-4, 4) = -1
    assert r64.idivup_c(-3, 4) == 1
    assert r64.idivup_c(-4, 4) == -1
    assert r64.idivup_c(-5, 4) == 0
    assert r64.idivup_c(5, 4) == 2
    assert r64.idivup_c(8, 4) == 2
