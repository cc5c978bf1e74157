"""Whole frame sequences through FrameStep against the same sequence chained
on the reference's own CUDA kernels (oracle/reference_step.py), and against
the CPU oracle, compared op by op on identical inputs.

Identical inputs: each frame, FrameStep starts from the reference chain's
history (out_log, ols1, ols2, linearZ, normal of the previous frame), and the
regression's outputs that the rest of FrameStep consumes are replaced by the
reference's.  The regression itself is compared separately, on the
reference's own log inputs and as FrameStep computed it.  So a last-bit
difference in one op cannot turn a near-tie in a later op (temporal
screening compares neighbourhood minima and maxima) into a different
decision, and every op downstream is held to its own bar:

  * bit-exact: the reprojection mask, the three reprojected buffers, the
    eroded mask, all four temporal-screening outputs, and (plain path) the
    spatial filter's sums and weight sums;
  * rtol 1e-4: the regression outputs (absolute floor 1e-5: outputs the
    reference clamps at zero), the denoised frame, its log and the history
    (absolute floor 1e-6 of the frame's largest value), the aggregation
    gradients and dL/dalpha (floor 1e-6 of the largest magnitude), dL/dband
    (floor 1e-5 of the largest magnitude: sums of 121 taps of both signs);
    the average loss within rtol 1e-5;
  * log1p within 2 ulp (rtol 4e-7).

Workloads: 8 consecutive 256x256 frames (regression window 15, sparsity 4,
filter window 11, temporal screening 7/1) on the plain and the fused step;
10 consecutive 1920x1080 frames with per-cell motion at regression windows
15 and 17 (the reference's default) on the fused step; 4 frames of 96x128
against the CPU oracle.
"""
import numpy as np
import pytest
import torch

from gpu_util import needs_reference
from oracle import oracle as orc
from oracle.reference_step import ReferenceStep, aggregation_forward_backward

pytestmark = pytest.mark.gpu

SPIED = ("prepare_input", "cross_regression", "Reproject", "erode3x3", "temporal_screening",
         "erode_temporal_screening", "spatial_filter", "aggregation_loss", "spatial_filter_grad",
         "filter_aggregate")


class Checker:
    """Collects every mismatch of a frame so one run reports all of them."""

    def __init__(self):
        self.fails = []

    def equal(self, a, b, what):
        a, b = torch.as_tensor(a).detach(), torch.as_tensor(b).detach().to(a.device)
        if a.shape != b.shape:
            self.fails.append(f"{what}: shape {tuple(a.shape)} != {tuple(b.shape)}")
            return
        ne = a != b
        if a.is_floating_point():
            ne &= ~(torch.isnan(a) & torch.isnan(b))
        n = int(ne.sum())
        if n:
            self.fails.append(f"{what}: {n}/{ne.numel()} values differ")

    def close(self, a, b, what, rtol=1e-4, atol=1e-6):
        a = torch.as_tensor(a).detach().double()
        b = torch.as_tensor(b).detach().double().to(a.device)
        if a.shape != b.shape:
            self.fails.append(f"{what}: shape {tuple(a.shape)} != {tuple(b.shape)}")
            return
        fin = torch.isfinite(b)
        if not torch.equal(torch.isfinite(a), fin):
            self.fails.append(f"{what}: non-finite pattern differs")
            return
        d = torch.where(fin, (a - b).abs(), torch.zeros_like(a))
        bad = d > atol + rtol * b.abs()
        n = int(bad.sum())
        if n:
            rel = (d / b.abs().clamp_min(1e-30))[bad].max()
            self.fails.append(f"{what}: {n}/{bad.numel()} outside rtol {rtol:g} atol {atol:g}; "
                              f"max |diff| {float(d.max()):.3g}, max rel {float(rel):.3g}")

    def scaled(self, a, b, what, floor=1e-6, rtol=1e-4):
        self.close(a, b, what, rtol=rtol, atol=floor * float(torch.as_tensor(b).abs().max()))

    def done(self, where):
        assert not self.fails, where + ":\n  " + "\n  ".join(self.fails)


def run_spied(cd, monkeypatch, st, frame, ols=None):
    """One FrameStep call with every op it calls recorded (name -> outputs);
    with `ols`, the regression's (outa, outb) handed on are replaced by it."""
    seen = {}
    real = {n: getattr(cd.ops, n) for n in SPIED}

    def wrap(name):
        def f(*a, **k):
            r = real[name](*a, **k)
            seen[name] = r
            if name == "cross_regression" and ols is not None:
                return (ols[0], ols[1], r[2], r[3])
            return r
        return f

    with monkeypatch.context() as m:
        for n in SPIED:
            m.setattr(cd.ops, n, wrap(n))
        out = st(frame)
    return out, seen


def history_of(cd, h):
    return cd.step.History(h.out_log.clone(), h.ols1.clone(), h.ols2.clone(), h.linearZ.clone(),
                           h.normal.clone())


def check_frame(cd, chk, r, o, seen, cfg, frame, t):
    """Every op of one FrameStep frame against the reference chain's frame r."""
    y1, y2 = seen["prepare_input"]
    chk.close(y1, r["y1"], f"{t} log1p(color)", rtol=4e-7, atol=0)
    chk.close(y2, r["y2"], f"{t} log1p(color2)", rtol=4e-7, atol=0)
    # the regression on the reference's own inputs, and as the step ran it
    mine = cd.ops.cross_regression(r["y1"], r["y2"], frame["albedo"], frame["normal"],
                                   win_size=cfg.regression_width, sparsity=cfg.sparsity)
    step_reg = seen["cross_regression"]
    for i, nm in ((0, "ols1"), (1, "ols2")):
        chk.close(mine[i], r[nm], f"{t} regression {nm}", atol=1e-5)
        chk.close(step_reg[i], r[nm], f"{t} regression {nm} (step inputs)", atol=1e-5)
    succ, rep = seen["Reproject"]
    chk.equal(succ, r["success"], f"{t} reprojection mask")
    for i in range(3):
        chk.equal(rep[i], r["reprojected"][i], f"{t} reprojected buffer {i}")
    if cfg.fused:
        po, p1, p2, sp, ero = seen["erode_temporal_screening"]
    else:
        ero = seen["erode3x3"]
        po, p1, p2, sp = seen["temporal_screening"]
    chk.equal(ero, r["eroded"], f"{t} eroded mask")
    for a, k in ((po, "prev_out"), (p1, "prev_ols1"), (p2, "prev_ols2"), (sp, "success_prev")):
        chk.equal(a, r[k], f"{t} temporal screening {k}")
    if not cfg.fused:
        s1, s2, w1, w2 = seen["spatial_filter"]
        for a, k in ((s1, "sum1"), (s2, "sum2"), (w1, "sumw1"), (w2, "sumw2")):
            chk.equal(a, r[k], f"{t} spatial filter {k}")
        agg = seen["aggregation_loss"]
        for a, k in zip(agg[4:8], ("g_sum1", "g_sumw1", "g_sum2", "g_sumw2")):
            chk.scaled(a, r[k], f"{t} aggregation {k}")
    chk.scaled(o["out_log"], r["out_log"], f"{t} out_log")
    chk.scaled(o["out"], r["out"], f"{t} out")
    chk.close(o["avg_loss"], r["avg_loss"], f"{t} avg_loss", rtol=1e-5, atol=0)
    chk.scaled(o["g_alpha"], r["g_alpha"], f"{t} g_alpha")
    chk.scaled(o["g_band"], r["g_band"], f"{t} g_band", floor=1e-5)


def run_chain(cd, monkeypatch, H, W, n, seed, fused, win, motion):
    dev = torch.device("cuda:0")
    seq = cd.synth.make_sequence(H, W, seed=seed, object_motion=motion, device=dev, max_frames=n + 2)
    g = torch.Generator(device=dev).manual_seed(seed + 1)
    band = cd.synth.random_band((1, H, W), g, device=dev)
    alpha = torch.sigmoid(torch.randn((1, H, W, 1), generator=g, device=dev))
    cfg = cd.step.StepConfig(regression_width=win, filter_width=11, sparsity=4, win_curr=7, win_prev=1,
                             fused=fused)
    ref = ReferenceStep(win, 4, 11, 7, 1, band, alpha)
    st = cd.step.FrameStep(cfg)
    st.set_fixed_prediction(band, alpha)
    decisions = 0
    for t in range(n):
        f = {k: v for k, v in seq.frame(t).items() if k in cd.synth.FRAME_INPUTS}
        if ref.history is not None:
            st.history = history_of(cd, ref.history)
        r = ref(f)
        o, seen = run_spied(cd, monkeypatch, st, f, ols=(r["ols1"], r["ols2"]))
        torch.cuda.synchronize()
        chk = Checker()
        check_frame(cd, chk, r, o, seen, cfg, f, t)
        chk.done(f"{W}x{H} {'fused' if fused else 'plain'} win {win} frame {t}")
        decisions += int(r["success_prev"].sum())
    # the chain exercised both screening outcomes and real reprojection
    assert 0 < decisions < n * H * W


@needs_reference
@pytest.mark.parametrize("fused", [False, True], ids=["plain", "fused"])
def test_chain_256_vs_reference_kernels(cd, cuda, monkeypatch, fused):
    run_chain(cd, monkeypatch, 256, 256, 8, seed=2024, fused=fused, win=15, motion=0.0)


@needs_reference
@pytest.mark.parametrize("win", [15, 17])
def test_chain_1080p_vs_reference_kernels(cd, cuda, monkeypatch, win):
    run_chain(cd, monkeypatch, 1080, 1920, 10, seed=7 + win, fused=True, win=win, motion=4.0)


def test_chain_vs_cpu_oracle(cd, cuda, monkeypatch):
    """Four frames of the plain step against the oracle's ops on the CPU,
    op by op on identical inputs (the oracle's history and regression
    outputs): bit-exact masks and screening, FP32 outputs within 1e-4."""
    H, W = 96, 128
    dev = torch.device("cuda:0")
    seq = cd.synth.make_sequence(H, W, seed=8, object_motion=2.0)
    band = cd.synth.random_band((1, H, W), torch.Generator().manual_seed(2))
    alpha = torch.full((1, H, W, 1), 0.6)
    cfg = cd.step.StepConfig(regression_width=15)
    st = cd.step.FrameStep(cfg)
    st.set_fixed_prediction(band.to(dev), alpha.to(dev))
    z3 = np.zeros((1, H, W, 3), np.float32)
    hist = dict(out_log=z3, ols1=z3, ols2=z3, linz=z3, nrm=z3)
    one = np.ones((1, H, W, 1), np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    for t in range(4):
        fr = {k: v.numpy() for k, v in seq.frame(t).items()}
        y1, y2 = np.log1p(fr["color"]), np.log1p(fr["color2"])
        o1, o2, _, _ = orc.cross_regression(y1, y2, fr["albedo"], fr["normal"], 15, 4, 1)
        s, rep = orc.reproject(fr["mvec"], [hist["out_log"], hist["ols1"], hist["ols2"]], fr["linearZ"],
                               hist["linz"], fr["normal"], hist["nrm"], fr["pnFwidth"], one, one)
        ero = orc.erode3x3(s)
        po, p1, p2, sp = orc.temporal_screening(o1, o2, rep[0], rep[1], rep[2], ero, 7, 1)
        s1, s2, w1, w2 = orc.spatial_filter(o1, o2, fr["albedo"], fr["normal"], band.numpy(), 11)
        tt = torch.from_numpy
        agg = aggregation_forward_backward(tt(s1), tt(w1), tt(s2), tt(w2), alpha, tt(ero), tt(sp), tt(po),
                                           tt(fr["opacity"]), tt(o2), tt(o1), tt(p2), tt(p1))
        st.history = cd.step.History(*(T(a) for a in (hist["out_log"], hist["ols1"], hist["ols2"], hist["linz"],
                                                      hist["nrm"])))
        o, seen = run_spied(cd, monkeypatch, st, {k: T(v) for k, v in fr.items()}, ols=(T(o1), T(o2)))
        torch.cuda.synchronize()
        chk = Checker()
        reg = seen["cross_regression"]
        chk.close(reg[0], o1, f"{t} regression ols1", atol=1e-5)
        chk.close(reg[1], o2, f"{t} regression ols2", atol=1e-5)
        succ, rp = seen["Reproject"]
        chk.equal(succ, s, f"{t} reprojection mask")
        for i in range(3):
            chk.equal(rp[i], rep[i], f"{t} reprojected buffer {i}")
        chk.equal(seen["erode3x3"], ero, f"{t} eroded mask")
        for a, b, k in zip(seen["temporal_screening"], (po, p1, p2, sp), ("prev_out", "prev_ols1", "prev_ols2",
                                                                          "success_prev")):
            chk.equal(a, b, f"{t} temporal screening {k}")
        for a, b, k in zip(seen["spatial_filter"], (s1, s2, w1, w2), ("sum1", "sum2", "sumw1", "sumw2")):
            chk.scaled(a, b, f"{t} spatial filter {k}")
        chk.scaled(o["out_log"], agg[0], f"{t} out_log")
        chk.scaled(o["out"], agg[1], f"{t} out")
        chk.close(o["avg_loss"], agg[3], f"{t} avg_loss", rtol=1e-5, atol=0)
        chk.done(f"oracle chain frame {t}")
        hist = dict(out_log=agg[0].numpy(), ols1=o1, ols2=o2, linz=fr["linearZ"], nrm=fr["normal"])
