"""The rest of the frame step on the GPU: input preparation, the aggregation
loss forward/backward against its eager PyTorch FP32 restatement and FP64,
the fused filter + loss + gradient kernel against the plain op sequence,
plain against fused frame steps, overlapped training and the host-frame
pipeline.  Whole sequences against the reference and the oracle are in
test_gpu_chain.py."""
import numpy as np
import pytest
import torch

from gpu_util import N, T, frames
from helpers import assert_close, assert_equal
from oracle.reference_step import aggregation_forward_backward

pytestmark = pytest.mark.gpu


def test_prepare_input(cd, cuda):
    _, f = frames(cd, 64, 96, seed=1)
    y1, y2 = cd.ops.prepare_input(T(f["color"]), T(f["color2"]))
    assert_close(N(y1), np.log1p(f["color"]), "y1", rtol=4e-7, atol=0)   # 2 ulp
    assert_close(N(y2), np.log1p(f["color2"]), "y2", rtol=4e-7, atol=0)


@pytest.mark.parametrize("H,W", [(5, 7), (9, 13)])
def test_prepare_input_odd_sizes(cd, cuda, H, W):
    """3 x H x W not a multiple of 4: the scalar log1p kernel."""
    _, f = frames(cd, H, W, seed=2)
    y1, y2 = cd.ops.prepare_input(T(f["color"]), T(f["color2"]))
    assert_close(N(y1), np.log1p(f["color"]), "y1", rtol=4e-7, atol=0)
    assert_close(N(y2), np.log1p(f["color2"]), "y2", rtol=4e-7, atol=0)


def agg_inputs(H, W, B, seed, device):
    g = torch.Generator(device="cpu").manual_seed(seed)
    r = lambda c, lo=0.0, hi=1.0: (lo + (hi - lo) * torch.rand((B, H, W, c), generator=g)).to(device)
    w1, w2 = r(1, 0.5, 30.0), r(1, 0.5, 30.0)
    s1, s2 = r(3, 0, 3) * w1, r(3, 0, 3) * w2
    succ = (r(1) > 0.2).float()
    sp = (r(1) > 0.3).float()
    opac = (r(1) > 0.05).float()
    return [s1, w1, s2, w2, r(1), succ, sp, r(3, 0, 3), opac, r(3, 0, 3), r(3, 0, 3), r(3, 0, 3), r(3, 0, 3)]


@pytest.mark.parametrize("H,W,B", [(64, 96, 1), (37, 53, 2), (270, 480, 1)])
def test_aggregation_vs_torch_and_fp64(cd, cuda, H, W, B):
    x = agg_inputs(H, W, B, seed=H, device=cuda)
    mine = cd.ops.aggregation_loss(*x)
    ref32 = aggregation_forward_backward(*x)
    ref64 = aggregation_forward_backward(*[t.double() for t in x])
    names = ("out_log", "out", "loss", "avg_loss", "g_sum1", "g_sumw1", "g_sum2", "g_sumw2", "g_alpha")
    for m, r32, r64, nm in zip(mine, ref32, ref64, names):
        scale = float(r64.abs().max())
        assert_close(N(m), N(r32), nm + " vs torch fp32", atol=1e-6 * scale)
        assert_close(N(m), N(r64), nm + " vs fp64", atol=1e-6 * scale)
    again = cd.ops.aggregation_loss(*x)
    assert float(again[3]) == float(mine[3]), "the mean is reduced in a fixed order"


def filter_inputs(cd, H, W, seed, device):
    _, f = frames(cd, H, W, seed=seed)
    y1, y2 = np.log1p(f["color"]), np.log1p(f["color2"])
    g = torch.Generator().manual_seed(seed)
    band = cd.synth.random_band((1, H, W), g)
    x = agg_inputs(H, W, 1, seed, device)
    alpha, succ, sp, prev, opac, pl1, pl2 = x[4], x[5], x[6], x[7], x[8], x[11], x[12]
    return (T(y1), T(y2), T(f["albedo"]), T(f["normal"]), band.to(device), alpha, succ, sp, prev, opac, pl2, pl1)


@pytest.mark.parametrize("win", [11, 7])
def test_filter_aggregate_equals_plain_sequence(cd, cuda, win):
    ols1, ols2, alb, nrm, band, alpha, succ, sp, prev, opac, prev_ols1, prev_ols2 = filter_inputs(cd, 96, 128, win, cuda)
    fused = cd.ops.filter_aggregate(ols1, ols2, alb, nrm, band, alpha, succ, sp, prev, opac, prev_ols1, prev_ols2, win)
    s1, s2, w1, w2 = cd.ops.spatial_filter(ols1, ols2, alb, nrm, band, win_size=win)
    agg = cd.ops.aggregation_loss(s1, w1, s2, w2, alpha, succ, sp, prev, opac, ols2, ols1, prev_ols2, prev_ols1)
    gb = cd.ops.spatial_filter_grad(agg[4], agg[6], agg[5], agg[7], ols1, ols2, alb, nrm, band, win_size=win)
    torch.cuda.synchronize()
    # the fused kernel's weights are 2^(e log2 e) on ex2.approx.ftz, the plain
    # kernels' __expf: equal wherever the weight is a normal float, so the
    # sums differ at most by the contributions of weights below 2^-126
    for i, j, nm in ((0, 0, "out_log"), (1, 1, "out"), (3, None, "grad_band"), (4, 8, "grad_alpha")):
        assert_close(N(fused[i]), N(agg[j] if j is not None else gb), nm, rtol=1e-6, atol=1e-30)
    assert abs(float(fused[2]) - float(agg[3])) <= 1e-6 * abs(float(agg[3])), "avg_loss"


def test_plain_and_fused_steps_agree(cd, cuda):
    """Four frames of the plain and the fused step, the fused one started
    each frame from the plain one's history (identical inputs): the same
    masks and screening, the other outputs equal up to the contributions of
    subnormal filter weights (see test_filter_aggregate_equals_plain_sequence)."""
    H, W = 128, 192
    seq = cd.synth.make_sequence(H, W, seed=4, object_motion=2.0)
    band = cd.synth.random_band((1, H, W), torch.Generator().manual_seed(1)).to(cuda)
    alpha = torch.full((1, H, W, 1), 0.7, device=cuda)
    steps = []
    for fused in (False, True):
        st = cd.step.FrameStep(cd.step.StepConfig(regression_width=15, fused=fused))
        st.set_fixed_prediction(band, alpha)
        steps.append(st)
    plain, fused = steps
    for t in range(4):
        f = {k: v.to(cuda) for k, v in seq.frame(t).items()}
        if plain.history is not None:
            h = plain.history
            fused.history = cd.step.History(*(x.clone() for x in (h.out_log, h.ols1, h.ols2, h.linearZ, h.normal)))
        a, b = plain(f), fused(f)
        torch.cuda.synchronize()
        assert_equal(N(a["success"]), N(b["success"]), f"frame {t} success")
        for k in ("ols1", "ols2"):
            assert_equal(N(a[k]), N(b[k]), f"frame {t} {k}")
        for k in ("out_log", "out", "g_band", "g_alpha"):
            assert_close(N(b[k]), N(a[k]), f"frame {t} {k}", rtol=1e-6, atol=1e-30)
        assert abs(float(a["avg_loss"]) - float(b["avg_loss"])) <= 1e-6 * abs(float(a["avg_loss"]))


def _unet_frames(cd, H, W, seed, n, cuda):
    seq = cd.synth.make_sequence(H, W, seed=seed, object_motion=2.0)
    return [{k: v.to(cuda) for k, v in seq.frame(t).items() if k in cd.synth.FRAME_INPUTS} for t in range(n)]


def test_overlapped_training_equals_serial(cd, cuda):
    """The training update on its own stream, overlapping the next frame's
    pre-network ops, gives the same frames, losses and network parameters as
    the serial order (bit-identical: every kernel is deterministic)."""
    H, W = 96, 128
    fr = _unet_frames(cd, H, W, 21, 5, cuda)
    runs = []
    for overlap in (False, True):
        net = cd.unet.UNet(cuda, seed=3)
        st = cd.step.FrameStep(cd.step.StepConfig(regression_width=9, filter_width=7, fused=True,
                                                  overlap_training=overlap),
                               predictor=net, on_gradients=net.on_gradients)
        outs = [st(f) for f in fr]
        st.wait_training()
        torch.cuda.synchronize()
        runs.append(([N(o["out"]) for o in outs], [float(o["avg_loss"]) for o in outs], N(net.params)))
    (o0, l0, p0), (o1, l1, p1) = runs
    for t, (a, b) in enumerate(zip(o0, o1)):
        assert_equal(a, b, f"frame {t} out")
    assert l0 == l1
    assert_equal(p0, p1, "parameters after 5 updates")


def test_host_pipeline_equals_device_step(cd, cuda):
    """Frames from pinned host memory through HostFramePipeline (uploads and
    read-backs on copy streams) give the same denoised frames and losses as
    the step on device-resident inputs."""
    H, W = 64, 96
    fr = _unet_frames(cd, H, W, 22, 6, cuda)
    band = cd.synth.random_band((1, H, W), torch.Generator().manual_seed(5)).to(cuda)
    alpha = torch.full((1, H, W, 1), 0.6, device=cuda)
    cfg = cd.step.StepConfig(regression_width=9, filter_width=7, fused=True)
    ref = cd.step.FrameStep(cfg)
    ref.set_fixed_prediction(band, alpha)
    want = [ref(f) for f in fr]
    want = [(N(o["out"]), float(o["avg_loss"])) for o in want]
    st = cd.step.FrameStep(cfg)
    st.set_fixed_prediction(band, alpha)
    pipe = cd.step.HostFramePipeline(st, cuda)
    host = [{k: v.cpu().pin_memory() for k, v in f.items()} for f in fr]
    for t, h in enumerate(host):
        out, loss, ev = pipe(h)
        ev.synchronize()
        assert_equal(out.numpy(), want[t][0], f"frame {t} out")
        assert float(loss) == want[t][1]
    # back to back (copies overlapping the steps): the last two results
    st2 = cd.step.FrameStep(cfg)
    st2.set_fixed_prediction(band, alpha)
    pipe2 = cd.step.HostFramePipeline(st2, cuda)
    got = [pipe2(h) for h in host]
    torch.cuda.synchronize()
    for t in (len(host) - 2, len(host) - 1):
        got[t][2].synchronize()
        assert_equal(got[t][0].numpy(), want[t][0], f"frame {t} out (overlapped)")
        assert float(got[t][1]) == want[t][1]


def test_npy_sequence_through_host_pipeline(cd, cuda, tmp_path):
    """Frames written in the reference's NPY scene layout and read back by
    frames.NpySequence (pinned, read ahead on a thread) denoise through
    HostFramePipeline exactly as the same frames resident on the device."""
    H, W = 64, 96
    seq = cd.synth.make_sequence(H, W, seed=23, object_motion=2.0)
    fr = [{k: v for k, v in seq.frame(t).items() if k in cd.frames.STEP_TYPES} for t in range(4)]
    cd.frames.save_npy_sequence(str(tmp_path), fr)
    band = cd.synth.random_band((1, H, W), torch.Generator().manual_seed(6)).to(cuda)
    alpha = torch.full((1, H, W, 1), 0.6, device=cuda)
    cfg = cd.step.StepConfig(regression_width=9, filter_width=7, fused=True)
    ref = cd.step.FrameStep(cfg)
    ref.set_fixed_prediction(band, alpha)
    want = [N(ref({k: v.to(cuda) for k, v in f.items()})["out"]) for f in fr]
    st = cd.step.FrameStep(cfg)
    st.set_fixed_prediction(band, alpha)
    pipe = cd.step.HostFramePipeline(st, cuda)
    for t, f in cd.frames.NpySequence(str(tmp_path)).prefetch(depth=2):
        out, loss, ev = pipe(f)
        ev.synchronize()
        assert_equal(out.numpy(), want[t], f"frame {t} out")
