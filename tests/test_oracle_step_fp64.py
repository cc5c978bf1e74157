"""The float64 full-step restatement (oracle/step_fp64.py) used by the
precision report: it runs a short sequence on the CPU, and its
aggregation + filter autograd gradient of dL/dband equals the closed-form
aggregation gradient pushed through the filter by autograd alone."""
import numpy as np
import torch

from oracle import step_fp64 as s64
from oracle.reference_step import aggregation_forward_backward


def test_runs_and_learns(cd):
    H, W = 16, 24
    seq = cd.synth.make_sequence(H, W, seed=4)
    st = s64.StepFP64(cd.unet.glorot_init(2))
    p0 = st.p.clone()
    for t in range(2):
        f = {k: v.numpy() for k, v in seq.frame(t).items()}
        o = st(f)
        for k in ("ols1", "ols2", "band", "alpha", "out_log", "out", "g_band", "params"):
            assert np.isfinite(o[k]).all(), k
        assert o["band"].shape == (1, H, W, 5) and o["alpha"].shape == (1, H, W, 1)
        assert np.isfinite(o["avg_loss"]) and o["avg_loss"] > 0
    assert st.step == 2 and not torch.equal(st.p, p0)


def test_aggregation_gradient_matches_closed_form(cd):
    g = torch.Generator().manual_seed(0)
    B, H, W = 1, 6, 7
    r = lambda c: torch.rand((B, H, W, c), generator=g, dtype=torch.float64)
    s1, s2 = r(3) * 3, r(3) * 3
    w1, w2 = r(1) + 0.5, r(1) + 0.5
    alpha = r(1).requires_grad_(True)
    sums = [t.requires_grad_(True) for t in (s1, w1, s2, w2)]
    succ, succp = (r(1) > 0.3).double(), (r(1) > 0.3).double()
    prev, op = r(3), torch.ones((B, H, W, 1), dtype=torch.float64)
    l1, l2, p1, p2 = r(3), r(3), r(3), r(3)
    _, _, _, avg = s64.aggregation_fp64(sums[0], sums[1], sums[2], sums[3], alpha, succ, succp, prev, op,
                                        l1, l2, p1, p2)
    avg.backward()
    ref = aggregation_forward_backward(s1.detach(), w1.detach(), s2.detach(), w2.detach(), alpha.detach(),
                                    succ, succp, prev, op, l1, l2, p1, p2)
    for got, want in zip([sums[0].grad, sums[1].grad, sums[2].grad, sums[3].grad, alpha.grad], ref[4:9]):
        torch.testing.assert_close(got, want, rtol=1e-10, atol=1e-14)
