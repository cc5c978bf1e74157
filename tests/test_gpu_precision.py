"""Precision report: the full step on the GPU (FP32 ops, bf16 tensor-core
U-Net, online Adam) against the float64 restatement of the whole step
(oracle/step_fp64.py), frame by frame on a short 96x128 sequence.

Per output the report prints the max and mean relative error (relative to
max(|ref|, 1e-3 max|ref|)); the test bounds what the design promises:
  regression outputs (FP32 op on the FP32 log1p of the frame; the FP64
  restatement takes log1p in double): max rel <= 1e-3 (op parity on
  identical inputs, 1e-4, is tested against the reference kernels)
  denoised output (log space), alpha:        max err <= 5e-2 of max|ref|
  average loss:                              rel <= 5e-2
  parameter update direction:                cosine >= 0.9
and counts the FP64 Cholesky fallbacks per frame at cond_limit 1e6."""
import json

import numpy as np
import pytest
import torch

from oracle import step_fp64 as s64

pytestmark = pytest.mark.gpu
H, W, FRAMES = 96, 128, 3


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = np.maximum(np.abs(b), 1e-3 * max(np.abs(b).max(), 1e-30))
    r = np.abs(a - b) / scale
    return float(r.max()), float(r.mean())


def test_full_step_precision_report(cd, cuda, capsys):
    seq = cd.synth.make_sequence(H, W, seed=9, object_motion=4.0)
    frames = [{k: v for k, v in seq.frame(t).items() if k in cd.synth.FRAME_INPUTS} for t in range(FRAMES)]
    p0 = cd.unet.glorot_init(11)
    net = cd.unet.UNet("cuda:0", params=p0)
    cfg = cd.step.StepConfig(fused=True, fp64_cond_limit=1e6)
    step = cd.step.FrameStep(cfg, predictor=net, on_gradients=net.on_gradients)
    ref = s64.StepFP64(p0, regression_width=cfg.regression_width, filter_width=cfg.filter_width,
                       sparsity=cfg.sparsity)
    report = []
    prev_p, prev_r = p0.astype(np.float64), p0.astype(np.float64)
    for t, f in enumerate(frames):
        o = step({k: v.to("cuda:0") for k, v in f.items()})
        torch.cuda.synchronize()
        r = ref({k: v.numpy() for k, v in f.items()})
        got_p = net.params.cpu().numpy().astype(np.float64)
        du, dr = got_p - prev_p, r["params"] - prev_r
        prev_p, prev_r = got_p, r["params"]
        row = {"frame": t, "fp64_fallbacks": int(o["fp64_fallbacks"].item())}
        for k in ("ols1", "ols2", "alpha", "out_log", "out"):
            row[k] = rel(o[k].cpu().numpy(), r[k])
        row["inv_band"] = rel(1.0 / o["band"].cpu().numpy(), 1.0 / r["band"])
        row["avg_loss"] = abs(float(o["avg_loss"]) - r["avg_loss"]) / abs(r["avg_loss"])
        row["update_cosine"] = float(du @ dr / (np.linalg.norm(du) * np.linalg.norm(dr)))
        report.append(row)
        assert row["ols1"][0] <= 1e-3 and row["ols2"][0] <= 1e-3, row
        for k in ("alpha", "out_log"):
            err = np.abs(o[k].cpu().numpy() - r[k]).max() / np.abs(r[k]).max()
            assert err <= 5e-2, (k, err, row)
        assert row["avg_loss"] <= 5e-2, row
        assert row["update_cosine"] >= 0.9, row
    with capsys.disabled():
        print("\nprecision report (max rel, mean rel per output):")
        for row in report:
            print(json.dumps(row))
