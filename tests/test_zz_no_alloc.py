"""cd_cross_regression_noalloc: cross-regression for callers that cannot
allocate device memory while the op runs (an engine frame loop that owns all
device memory and forbids mid-frame allocations, a plugin host that gives
plugins no allocator).  Its scratch is a fixed device array inside the
library instead of a caller workspace.

The test calls it through the C ABI with ctypes, twice in a row on different
frames, and checks each result against the regular entry point
(cd_cross_regression with a workspace, through the op surface) within the
parity tolerance of the other regression tests (rtol 1e-4, atol 1e-5); it
also checks that a frame too large for the array is refused.  It is collected
last (file name) and runs the same alone or after the other tests."""
import ctypes

import numpy as np
import pytest
import torch

from helpers import assert_close

pytestmark = pytest.mark.gpu


def _call_noalloc(cd, ins, win, sp, rs):
    L = cd._lib.lib()
    imga = ins[0]
    B, H, W, _ = imga.shape
    outa = torch.empty((B, H // rs, W // rs, 3), dtype=torch.float32, device=imga.device)
    outb = torch.empty_like(outa)
    vara = torch.empty((B, H, W, 1), dtype=torch.float32, device=imga.device)
    varb = torch.empty_like(vara)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.cd_cross_regression_noalloc(*[p(t) for t in ins], p(outa), p(outb), p(vara), p(varb),
                                       B, H, W, win, sp, rs, st)
    return rc, (outa, outb, vara, varb)


def _frame(cd, H, W, seed, device):
    f = cd.synth.make_sequence(H, W, seed=seed, object_motion=2.0, device=device).frame(3)
    return [torch.log1p(f["color"]), torch.log1p(f["color2"]), f["albedo"], f["normal"]]


def test_noalloc_matches_workspace_entry_point(cd, cuda):
    L = cd._lib.lib()
    cap = L.cd_cross_regression_noalloc_capacity()
    assert cap == 40 << 20
    # two calls in a row: the second reuses the array the first left behind
    for H, W, win, sp, rs, seed in ((256, 320, 15, 4, 1, 1), (1080, 1920, 17, 4, 2, 2)):
        ins = _frame(cd, H, W, seed, cuda)
        assert L.cd_cross_regression_workspace_size(1, H, W, sp) <= cap
        rc, got = _call_noalloc(cd, ins, win, sp, rs)
        assert rc == 0, L.cd_get_last_error()
        want = cd.ops.cross_regression(*ins, win_size=win, sparsity=sp, recon_scale=rs)
        torch.cuda.synchronize()
        for g, w, nm in zip(got, want, ("outa", "outb", "vara", "varb")):
            assert_close(g.cpu().numpy(), w.cpu().numpy(), f"{H}x{W} {nm}", rtol=1e-4, atol=1e-5)


def test_noalloc_refuses_oversized_frames(cd, cuda):
    L = cd._lib.lib()
    H, W = 2160, 3840
    assert L.cd_cross_regression_workspace_size(1, H, W, 4) > L.cd_cross_regression_noalloc_capacity()
    x = torch.zeros((1, H, W, 3), device=cuda)
    rc, _ = _call_noalloc(cd, [x, x, x, x], 15, 4, 1)
    assert rc == cd._lib.CD_ENOMEM
    assert b"built-in array" in L.cd_get_last_error()
