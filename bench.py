#!/usr/bin/env python
"""Benchmark of the per-frame hot path of the online cross-regression denoiser.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

One step = one 1920x1080 frame of a seeded synthetic sequence through the
hot path in the reference's order (scripts/main.py:250-313): log1p,
cross_regression (win 15, sparsity 4), Reproject of the 3-tensor history,
3x3 erosion + temporal screening (7/1), spatial filter (win 11), the
aggregation loss forward and backward, spatial_filter_grad.  The network
that predicts band/alpha is not part of this step: band and alpha are fixed
seeded tensors.

Prints one JSON line.  `value` is frames/s of the fused path with every
frame's inputs already resident in HBM (182 MB of new inputs per frame, more
than the 126 MB L2, so no L2 flush is needed); `plain` is the drop-in op
sequence; `e2e` runs the same step through the public API from pinned host
buffers with the host->device copy of the frame's inputs and the
device->host read of the denoised frame inside the timed region.
`--impl reference` runs the same step on the reference's own CUDA kernels
(oracle/_ref, compiled from the reference sources).

Under torchrun (N > 1) every rank denoises its own stream (replicas, weak
scaling); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

cd = ge.load_package()
from cross_denoiser_b200 import ops, step as stepmod, synth  # noqa: E402

METRIC = ("1080p denoised frames/sec and p50/p99 ms/frame on 1 B200, chosen vs plain, "
          "at ≤1e-4 rel err")

# Algorithmic FP32 work per unit, counting a fused multiply-add as 2 FLOP and
# an exp or a division as 1 (the minimal formulation of each op):
#   regression: per window tap and buffer, 61 normal-equation updates (122),
#     9 weighted products, colour / albedo / normal differences, the weight
#     and the normalised colour feature (~19)                -> 150
#   block reconstruction: per (pixel, centre, buffer)          -> 55
#   variance: per pixel and buffer                             -> 20
#   spatial filter forward: per (pixel, tap), both buffers     -> 60
#   spatial filter gradient: per (pixel, tap), both buffers    -> 110
FLOP = {"regression_tap": 150, "recon_pair": 55, "variance_px": 20, "filter_tap": 60, "grad_tap": 110}
# Algorithmic HBM bytes per pixel (each input read once, each output written
# once): reprojection 153, erosion + temporal screening 104.
BYTES = {"reproject_px": 153, "temporal_px": 104}
# DRAM bytes (read + write) per launch of the dominant kernel at 1920x1080,
# filter window 11: dram__bytes_read.sum + dram__bytes_write.sum of one
# earlier ncu capture of this workload, not measured by this run (ncu is not
# available to it); reported as roofline.traffic with that provenance.
NCU_TRAFFIC = {"filter_aggregate": 327_517_696}


def args_parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--pool", type=int, default=24, help="distinct frames resident in HBM, cycled")
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--win", type=int, default=15)
    ap.add_argument("--filter-win", type=int, default=11)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--serve", action="store_true",
                    help="serving run: 16 mixed-resolution streams (4x720p, 8x1080p, 3x1440p, 1x2160p)")
    ap.add_argument("--serve-frames", type=int, default=30, help="frames per stream in the serving run")
    ap.add_argument("--no-serve", action="store_true", help="leave the serving run out of the default line")
    ap.add_argument("--ncu-region", choices=["fused", "full"], default=None,
                    help="bracket the timed steps of the fused ops step or of the full step (with the U-Net) "
                         "with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# frames
# ---------------------------------------------------------------------------
def make_frames(H, W, n, seed, device):
    seq = synth.make_sequence(H, W, seed=seed, object_motion=4.0, device=device, max_frames=max(n + 2, 8))
    keep = synth.FRAME_INPUTS
    return [{k: v for k, v in seq.frame(t).items() if k in keep} for t in range(n)]


def fixed_prediction(H, W, seed, device):
    g = torch.Generator(device=device).manual_seed(seed)
    band = synth.random_band((1, H, W), g, device=device)
    alpha = torch.sigmoid(torch.randn((1, H, W, 1), generator=g, device=device))
    return band, alpha


# ---------------------------------------------------------------------------
# timing helpers
# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        uuid = str(getattr(torch.cuda.get_device_properties(device), "uuid", ""))
        self.ident = ("GPU-" + uuid) if uuid and not uuid.startswith("GPU-") else (uuid or "0")
        self.proc, self.path = None, f"/tmp/cd_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.ident}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait()
            self.fh.close()

    def summary(self):
        if self.proc is None:
            return None
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7 and parts[0].isdigit():
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names[1:], r[3:]) if v.lower() == "active"})
        sm = [int(r[0]) for r in rows]
        return {"sm_mhz": int(statistics.median(sm)), "sm_max_mhz": int(rows[0][1]), "samples": len(rows),
                "reasons": reasons}


def timed_steps(fn, frames, warmup, steps, stream, per_op=None):
    """Run warmup + steps frames; per-step CUDA events on `stream`."""
    for t in range(warmup):
        fn(frames[t % len(frames)], t)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    ev[0].record(stream)
    for i in range(steps):
        fn(frames[(warmup + i) % len(frames)], warmup + i)
        ev[i + 1].record(stream)
    torch.cuda.synchronize()
    ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
    total = ev[0].elapsed_time(ev[-1])
    return total, ms


def timed_host_pipeline(pipe, host, warmup, steps, stream):
    """Frames from pinned host memory through a HostFramePipeline: the timed
    region starts before the first upload and ends after the last read-back.
    Returns the total ms and the intervals between consecutive read-backs."""
    for t in range(warmup):
        pipe(host[t % len(host)])
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pipe.up.wait_event(e0)
    pipe.down.wait_event(e0)
    marks = [e0]
    for i in range(steps):
        pipe(host[(warmup + i) % len(host)])
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(pipe.down)
        marks.append(ev)
    pipe.drain(stream)
    e1 = torch.cuda.Event(enable_timing=True)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), [marks[i].elapsed_time(marks[i + 1]) for i in range(steps)]


def timed_frame_latency(step, frames, warmup, steps, stream):
    """Frames back to back through a FrameStep whose training update may run
    on its own stream: the total time ends after the last update; the
    latency of a frame is from its first op to its denoised output."""
    for t in range(warmup):
        step(frames[t % len(frames)])
    step.wait_training(stream)
    torch.cuda.synchronize()
    starts, outs = [], []
    for i in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(frames[(warmup + i) % len(frames)])
        e1.record(stream)
        starts.append(e0)
        outs.append(e1)
    step.wait_training(stream)
    end = torch.cuda.Event(enable_timing=True)
    end.record(stream)
    torch.cuda.synchronize()
    return starts[0].elapsed_time(end), [s.elapsed_time(o) for s, o in zip(starts, outs)]


def pct(xs, q):
    return float(np.percentile(np.asarray(xs), q))


def max_over_ranks(x, world):
    from cross_denoiser_b200 import replicas
    return replicas.max_over_ranks(x) if world > 1 else x


# ---------------------------------------------------------------------------
# measurements of the product path
# ---------------------------------------------------------------------------
def op_timer(stepper, stream):
    """Wrap the ops the step calls so every call is bracketed by CUDA events."""
    names = ("prepare_input", "cross_regression", "Reproject", "erode3x3", "temporal_screening",
             "erode_temporal_screening", "spatial_filter", "aggregation_loss", "spatial_filter_grad",
             "filter_aggregate")
    store = {n: [] for n in names}
    orig = {n: getattr(ops, n) for n in names}

    def wrap(n):
        def f(*a, **k):
            # the op's own stream (the fused step runs Reproject on a side stream)
            st = torch.cuda.current_stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            r = orig[n](*a, **k)
            e1.record(st)
            store[n].append((e0, e1))
            return r
        return f

    class Ctx:
        def __enter__(self):
            for n in names:
                setattr(ops, n, wrap(n))
                setattr(stepmod.ops, n, getattr(ops, n))
            return store

        def __exit__(self, *exc):
            for n in names:
                setattr(ops, n, orig[n])

    return Ctx()


def fp32_peak(device):
    out = torch.empty(148 * 8 * 256, device=device)
    L = cd._lib.lib()
    import ctypes
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    iters = 4000
    for _ in range(2):
        cd._lib.check(L.cd_fp32_fma_probe(ctypes.c_void_p(out.data_ptr()), 148 * 8, iters, st), "fp32_fma_probe")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    cd._lib.check(L.cd_fp32_fma_probe(ctypes.c_void_p(out.data_ptr()), 148 * 8, iters, st), "fp32_fma_probe")
    e1.record()
    torch.cuda.synchronize()
    flop = 148 * 8 * 256 * iters * 128 * 2
    return flop / (e0.elapsed_time(e1) * 1e-3) / 1e12


def _centres_per_axis(n, hw, sp):
    """Centres each output position reconstructs from along one axis, with the
    reference's clamped iDivUp range (ops/regression.cu.cc:312-315)."""
    p = np.arange(n)
    a = p - hw
    lo = np.maximum(0, np.where(a % sp != 0, np.trunc(a / sp) + 1, a // sp).astype(np.int64))
    hi = np.minimum((n - 1) // sp, (p + hw) // sp)
    return np.maximum(hi - lo + 1, 0)


def regression_flop(H, W, win, sp):
    taps = (H // sp) * (W // sp) * win * win * 2
    pairs = int(_centres_per_axis(H, win // 2, sp).sum()) * int(_centres_per_axis(W, win // 2, sp).sum()) * 2
    return taps * FLOP["regression_tap"] + pairs * FLOP["recon_pair"] + 2 * H * W * FLOP["variance_px"]


def differentiation_costs(device, stream):
    """512x512, batch 4, radius 7: the spatial filter's band gradient by
    recomputation (this repository's design) against the reference's design
    (the forward stores 128 B/px of partials, the gradient reads them), and
    the regression backward, recomputing its forward or reusing a kept one:
    time per call and the extra device memory each needs beyond the op's
    inputs and outputs."""
    B, H, W, win = 4, 512, 512, 15
    frames = make_frames(H, W, 2, 77, device)
    f = frames[1]
    ia, ib = torch.log1p(f["color"]), torch.log1p(f["color2"])
    ia, ib, al, nr = [t.expand(B, -1, -1, -1).contiguous() for t in (ia, ib, f["albedo"], f["normal"])]
    g = torch.Generator(device=device).manual_seed(78)
    band = synth.random_band((B, H, W), g, device=device)
    gs = [torch.randn((B, H, W, c), generator=g, device=device) for c in (3, 3, 1, 1)]

    def timed(fn, n=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {"shape": [B, H, W], "window": win}
    fwd = timed(lambda: ops.spatial_filter(ia, ib, al, nr, band, win_size=win))
    grd = timed(lambda: ops.spatial_filter_grad(*gs, ia, ib, al, nr, band, win_size=win))
    part = ops.spatial_filter_stored(ia, ib, al, nr, band, win_size=win)[4]
    fwd_s = timed(lambda: ops.spatial_filter_stored(ia, ib, al, nr, band, win_size=win))
    grd_s = timed(lambda: ops.spatial_filter_grad_stored(*gs, part))
    out["filter_recompute"] = {"forward_ms": round(fwd, 4), "grad_ms": round(grd, 4), "extra_bytes": 0}
    out["filter_stored"] = {"forward_ms": round(fwd_s, 4), "grad_ms": round(grd_s, 4),
                            "extra_bytes": part.numel() * 4}
    y = [ia, ib, al, nr]
    rf = timed(lambda: ops.cross_regression(*y, win_size=win, sparsity=4), n=10)
    gu = [torch.randn((B, H, W, c), generator=g, device=device) for c in (3, 3, 1, 1)]
    rb = timed(lambda: ops.cross_regression_grad(*gu, *y, win, 4, 1), n=10)
    ws = cd._lib.lib().cd_cross_regression_grad_workspace_size(B, H, W, 4, 1)
    # the training pair: a forward that keeps its state, a backward that reuses it
    _, kept = ops.cross_regression_keep(*y, win, 4, 1)
    rfk = timed(lambda: ops.cross_regression_keep(*y, win, 4, 1), n=10)
    rbk = timed(lambda: ops.cross_regression_grad_kept(*gu, *y, win, 4, 1, kept), n=10)
    out["regression"] = {"forward_ms": round(rf, 4), "backward_ms": round(rb, 4), "backward_workspace_bytes": int(ws),
                         "forward_keep_ms": round(rfk, 4), "backward_kept_ms": round(rbk, 4)}
    return out


def unet_flop(H, W):
    """Tensor-core FLOP of one training step of the U-Net (forward + input and
    weight gradients of the 3x3 convolutions) at H x W, counting only the
    real channels (the kernels pad N to 16 and K to 16)."""
    convs = [(15, 8, 0), (8, 8, 0), (8, 16, 1), (16, 16, 1), (16, 32, 2), (32, 32, 2), (48, 16, 1),
             (16, 16, 1), (24, 8, 0)]
    fwd = sum(2 * 9 * ci * co * (H >> l) * (W >> l) for ci, co, l in convs)
    dgrad = fwd - 2 * 9 * 15 * 8 * H * W
    return {"forward": fwd, "backward": dgrad + fwd}


def cpu_baseline(H, W, win, fwin, seed):
    """The oracle (C, OpenMP over all host threads) on a bounded sample: whole
    1080p frames through the same op sequence, until ~10 s have elapsed."""
    from oracle import oracle as orc
    from oracle.reference_step import aggregation_forward_backward
    cores = len(os.sched_getaffinity(0))
    frames = make_frames(H, W, 3, seed, "cpu")
    f = [{k: v.numpy() for k, v in fr.items()} for fr in frames]
    g = torch.Generator().manual_seed(seed)
    band = synth.random_band((1, H, W), g).numpy()
    alpha = torch.sigmoid(torch.randn((1, H, W, 1), generator=g)).numpy()
    z3 = np.zeros((1, H, W, 3), np.float32)
    hist = dict(out_log=z3, ols1=z3, ols2=z3, linz=z3, nrm=z3)
    one = np.ones((1, H, W, 1), np.float32)
    done, t0 = 0, time.perf_counter()
    for fr in f[1:]:
        y1, y2 = np.log1p(fr["color"]), np.log1p(fr["color2"])
        o1, o2, _, _ = orc.cross_regression(y1, y2, fr["albedo"], fr["normal"], win, 4, 1)
        s, rep = orc.reproject(fr["mvec"], [hist["out_log"], hist["ols1"], hist["ols2"]], fr["linearZ"],
                               hist["linz"], fr["normal"], hist["nrm"], fr["pnFwidth"], one, one)
        ero = orc.erode3x3(s)
        po, p1, p2, sp = orc.temporal_screening(o1, o2, rep[0], rep[1], rep[2], ero, 7, 1)
        s1, s2, w1, w2, pa, pb = orc.spatial_filter(o1, o2, fr["albedo"], fr["normal"], band, fwin, partials=True)
        tt = lambda a: torch.from_numpy(a)
        agg = aggregation_forward_backward(tt(s1), tt(w1), tt(s2), tt(w2), tt(alpha), tt(ero), tt(sp),
                                           tt(po), tt(fr["opacity"]), tt(o2), tt(o1), tt(p2), tt(p1))
        orc.spatial_filter_grad_from_partials(*[a.numpy() for a in (agg[4], agg[6], agg[5], agg[7])], pa, pb)
        hist = dict(out_log=agg[0].numpy(), ols1=o1, ols2=o2, linz=fr["linearZ"], nrm=fr["normal"])
        done += 1
        if time.perf_counter() - t0 > 10.0:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "frames/s", "cores": cores, "kind": "port",
            "sample": f"{done} consecutive {W}x{H} frames through the full op sequence "
                      f"(regression win {win}, filter win {fwin}), {dt:.1f} s"}


def run_mine(a, rank, world, device):
    H, W = a.height, a.width
    n = min(a.pool, a.warmup + a.steps)
    frames = make_frames(H, W, n, a.seed + 7919 * rank, device)
    band, alpha = fixed_prediction(H, W, a.seed, device)
    stream = torch.cuda.current_stream()
    res = {}

    def stepper(fused, win):
        st = stepmod.FrameStep(stepmod.StepConfig(regression_width=win, filter_width=a.filter_win, fused=fused))
        st.set_fixed_prediction(band, alpha)
        return lambda f, t: st(f)

    clk = Clocks(device)
    with clk:
        # plain (drop-in op sequence)
        if world > 1:
            torch.distributed.barrier()
        with op_timer(None, stream) as store_plain:
            total, ms = timed_steps(stepper(False, a.win), frames, a.warmup, a.steps, stream)
        total = max_over_ranks(total, world)
        res["plain"] = {"value": world * a.steps / (total * 1e-3), "ms_per_step": total / a.steps,
                        "p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99)}

        # chosen (fused) path, with per-op events and the launch count
        cd._lib.LAUNCHES["count"] = 0
        fn = stepper(True, a.win)
        if world > 1:
            torch.distributed.barrier()
        if a.ncu_region == "fused":
            torch.cuda.profiler.start()
        with op_timer(fn, stream) as store:
            total, ms = timed_steps(fn, frames, a.warmup, a.steps, stream)
        if a.ncu_region == "fused":
            torch.cuda.profiler.stop()
        launches = cd._lib.LAUNCHES["count"] * a.steps // (a.steps + a.warmup)
        total = max_over_ranks(total, world)
        res["value"] = world * a.steps / (total * 1e-3)
        res["ms_per_step"] = total / a.steps
        res["p50_ms"], res["p99_ms"] = pct(ms, 50), pct(ms, 99)
        res["gpu_launches"] = launches
        per_op = {}
        for k, evs in store.items():
            evs = evs[a.warmup:] if len(evs) > a.warmup else evs
            if evs:
                per_op[k] = statistics.mean(e0.elapsed_time(e1) for e0, e1 in evs)
        res["per_op_ms"] = {k: round(v, 4) for k, v in per_op.items()}
        per_op_plain = {}
        for k, evs in store_plain.items():
            evs = evs[a.warmup:] if len(evs) > a.warmup else evs
            if evs:
                per_op_plain[k] = statistics.mean(e0.elapsed_time(e1) for e0, e1 in evs)
        res["plain"]["per_op_ms"] = {k: round(v, 4) for k, v in per_op_plain.items()}

        # end to end through the public API, from pinned host buffers: every
        # frame's inputs are uploaded and its denoised frame and loss read back
        # inside the timed region (HostFramePipeline overlaps both with the step)
        host = [{k: v.cpu().pin_memory() for k, v in frames[i].items()} for i in range(min(4, n))]
        st = stepmod.FrameStep(stepmod.StepConfig(regression_width=a.win, filter_width=a.filter_win, fused=True))
        st.set_fixed_prediction(band, alpha)
        pipe = stepmod.HostFramePipeline(st, device)
        if world > 1:
            torch.distributed.barrier()
        e2e_steps = max(1, min(a.steps, 40))
        e2e_total, e2e_ms = timed_host_pipeline(pipe, host, min(a.warmup, 4), e2e_steps, stream)
        e2e_total = max_over_ranks(e2e_total, world)
        h2d = sum(v.numel() * v.element_size() for v in host[0].values())
        res["e2e"] = {"value": world * e2e_steps / (e2e_total * 1e-3), "unit": "frames/s", "steps": e2e_steps,
                      "h2d_bytes_per_step": int(h2d),
                      "d2h_bytes_per_step": int(pipe.out_host[0].numel() * 4 + pipe.loss_host[0].numel() * 4),
                      "ms_per_step": e2e_total / e2e_steps, "p50_interval_ms": pct(e2e_ms, 50),
                      "p99_interval_ms": pct(e2e_ms, 99)}
        del pipe, host
        # full step: the fused ops plus the online-trained U-Net (forward,
        # backward through band/alpha, Adam), as the reference's train_step
        net = cd.unet.UNet(device, seed=a.seed)
        full = stepmod.FrameStep(stepmod.StepConfig(regression_width=a.win, filter_width=a.filter_win, fused=True),
                                 predictor=net, on_gradients=net.on_gradients)
        net_ev = {"unet_forward": [], "unet_backward": [], "adam_update": []}
        orig_m = {"unet_forward": net.forward, "unet_backward": net.backward, "adam_update": net.apply_gradients}

        def timed(name):
            def f(*args):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(torch.cuda.current_stream())
                r = orig_m[name](*args)
                e1.record(torch.cuda.current_stream())
                net_ev[name].append((e0, e1))
                return r
            return f
        net.forward, net.backward, net.apply_gradients = (timed("unet_forward"), timed("unet_backward"),
                                                          timed("adam_update"))
        full.predictor = net.forward
        if world > 1:
            torch.distributed.barrier()
        if a.ncu_region == "full":
            torch.cuda.profiler.start()
        total, ms = timed_steps(lambda f, t: full(f), frames, a.warmup, a.steps, stream)
        if a.ncu_region == "full":
            torch.cuda.profiler.stop()
        total = max_over_ranks(total, world)
        fo = {}
        for k, evs in net_ev.items():
            evs = evs[a.warmup:]
            if evs:
                fo[k] = round(statistics.mean(e0.elapsed_time(e1) for e0, e1 in evs), 4)
        # the same full step with the FP64 Cholesky fallback (condition estimate > 1e6):
        # fallbacks per frame and its time
        net2 = cd.unet.UNet(device, seed=a.seed)
        fb = stepmod.FrameStep(stepmod.StepConfig(regression_width=a.win, filter_width=a.filter_win, fused=True,
                                                  fp64_cond_limit=1e6),
                               predictor=net2, on_gradients=net2.on_gradients)
        counts = []
        kf = max(1, min(a.steps, 20))
        totf, _ = timed_steps(lambda f, t: counts.append(fb(f)["fp64_fallbacks"]), frames, 2, kf, stream)
        counts = [int(c.item()) for c in counts[2:]]
        fp64_fb = {"cond_limit": 1e6, "ms_per_step": totf / kf, "fallbacks_per_frame_mean": statistics.mean(counts),
                   "fallbacks_per_frame_max": max(counts),
                   "solves_per_frame": 2 * 3 * (H // 4) * (W // 4)}
        # the same full step with the training update (U-Net backward + Adam)
        # on its own stream, overlapping the next frame's regression,
        # reprojection and screening; latency = frame start -> denoised frame
        net3 = cd.unet.UNet(device, seed=a.seed)
        ov = stepmod.FrameStep(stepmod.StepConfig(regression_width=a.win, filter_width=a.filter_win, fused=True,
                                                  overlap_training=True),
                               predictor=net3, on_gradients=net3.on_gradients)
        if world > 1:
            torch.distributed.barrier()
        tot_o, lat_o = timed_frame_latency(ov, frames, a.warmup, a.steps, stream)
        tot_o = max_over_ranks(tot_o, world)
        res["full_step"] = {"value": world * a.steps / (tot_o * 1e-3), "unit": "frames/s",
                            "schedule": "training update overlapped with the next frame's pre-network ops",
                            "ms_per_step": tot_o / a.steps, "p50_ms": pct(lat_o, 50), "p99_ms": pct(lat_o, 99),
                            "latency": "frame start to denoised frame on the device",
                            "serial": {"value": world * a.steps / (total * 1e-3), "ms_per_step": total / a.steps,
                                       "p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99)},
                            "fp64_fallback": fp64_fb,
                            "network_ms": fo, "unet_error_flag": max(net.error_flag(), net3.error_flag()),
                            "unet_tensor_flop_per_frame": unet_flop(H, W)}
    res["clocks"] = clk.summary()

    res["differentiation"] = differentiation_costs(device, stream)

    # regression-width sweep (radius 5 / 7 / 9, and 8: the reference's default 17)
    if not a.no_sweep:
        res["sweep_frames_per_s"] = {}
        for win in (11, 15, 17, 19):
            k = max(1, min(a.steps, 50))
            total, _ = timed_steps(stepper(True, win), frames, 2, k, stream)
            res["sweep_frames_per_s"][f"win{win}"] = round(k / (total * 1e-3), 2)

    # roofline of the dominant kernel: the fused filter + aggregation kernel,
    # 44 % of the fused step's kernel time in the ncu launch list (the
    # cross_regression op is three kernels, and its event span in the fused
    # step also covers the Reproject it overlaps)
    peak = fp32_peak(device)
    dom = "filter_aggregate" if "filter_aggregate" in per_op else max(per_op, key=per_op.get)
    px = H * W
    flop = {"cross_regression": regression_flop(H, W, a.win, 4),
            "spatial_filter": px * a.filter_win ** 2 * FLOP["filter_tap"],
            "spatial_filter_grad": px * a.filter_win ** 2 * FLOP["grad_tap"],
            "filter_aggregate": px * a.filter_win ** 2 * FLOP["grad_tap"]}
    if dom in flop:
        ach = flop[dom] / (per_op[dom] * 1e-3) / 1e12
        res["roofline"] = {"kernel": dom, "bound": "fp32", "achieved": round(ach, 2), "peak": round(peak, 2),
                           "unit": "TFLOP/s", "frac": round(ach / peak, 3), "traffic": NCU_TRAFFIC.get(dom),
                           "peak_source": "measured FP32 FMA probe (cd_fp32_fma_probe) in this run",
                           "flop_per_launch": flop[dom]}
    hbm = 6547.5
    try:
        hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except (OSError, KeyError, ValueError):
        pass
    bw = {}
    # Reproject timed alone (the plain step; the fused step overlaps it with the regression)
    for k, per, src in (("Reproject", BYTES["reproject_px"], per_op_plain),
                        ("erode_temporal_screening", BYTES["temporal_px"], per_op)):
        if k in src:
            gbs = per * px / (src[k] * 1e-3) / 1e9
            bw[k] = {"achieved_gbs": round(gbs, 1), "peak_gbs": hbm, "frac": round(gbs / hbm, 3),
                     "ms": round(src[k], 4)}
    res["roofline_hbm"] = bw
    return res


SERVE_RES = [(720, 1280)] * 4 + [(1080, 1920)] * 8 + [(1440, 2560)] * 3 + [(2160, 3840)]


def run_serving(a, device):
    """Serving: 16 streams, each with its own sequence (seed), history and
    online-trained U-Net resident in HBM.  Chosen = continuous batching over
    per-stream CUDA streams with graph replay; plain = the eager drop-in step,
    one frame at a time in arrival order.  In both arms every stream is
    admitted and its first WARM frames run (allocations, graph capture)
    before the timed region; the timed region serves frames WARM .. F-1 of
    every stream, once with every frame ready at t = 0 (saturated: aggregate
    frames/s) and once under Poisson arrivals at 30-120 Hz per stream
    (latency from arrival, and service time from dispatch)."""
    from cross_denoiser_b200 import serve
    WARM = 2
    res = SERVE_RES
    seeds = [a.seed + 101 * i for i in range(len(res))]
    src = serve.device_frame_source(res, seeds, device, pool=2)
    for sid in range(len(res)):
        src(sid, 0)
    torch.cuda.synchronize()
    rates = np.random.default_rng(a.seed).uniform(30.0, 120.0, len(res)).tolist()
    F = max(a.serve_frames, WARM + 2)
    sched = [q for q in serve.poisson_schedule(rates, F, seed=a.seed) if q.frame >= WARM]
    t0 = min(q.arrival for q in sched)
    sched = [serve.Request(q.arrival - t0, q.stream_id, q.frame) for q in sched]
    free, _ = torch.cuda.mem_get_info(device)
    budget = int(0.8 * free)
    cfg = stepmod.StepConfig(regression_width=a.win, filter_width=a.filter_win, fused=True)
    out = {"streams": len(res), "frames_per_stream": F, "warm_frames_untimed": WARM,
           "rates_hz": [round(r, 1) for r in rates], "offered_frames_per_s": round(sum(rates), 1),
           "hbm_budget_gb": round(budget / 1e9, 1)}
    measured = None
    with Clocks(device) as clk:
        for mode in ("saturated", "poisson"):
            srv = serve.Server(res, src, device, budget, cfg=cfg, seed=a.seed)
            if measured is None:
                srv.calibrate(frames=2)
                measured = dict(srv.measured)
                out["footprint_gb"] = {f"{W}x{H}": round(v / 1e9, 2) for (H, W), v in measured.items()}
            srv.measured = measured
            out["resident_streams"] = srv.admit_all()
            srv.warm(WARM)
            out[f"chosen_{mode}"] = serve.summarize(srv.run(sched, F, realtime=mode == "poisson"), res)
            del srv
        # plain: eager drop-in op sequence plus the same network, one frame at a time
        plain_cfg = stepmod.StepConfig(regression_width=a.win, filter_width=a.filter_win, fused=False)
        for mode in ("saturated", "poisson"):
            streams = {}
            for sid in range(len(res)):
                net = cd.unet.UNet(device, seed=a.seed + sid)
                streams[sid] = stepmod.FrameStep(plain_cfg, predictor=net, on_gradients=net.on_gradients)
                for t in range(WARM):
                    streams[sid](src(sid, t))
            torch.cuda.synchronize()
            results = []
            t0 = time.perf_counter()
            for q in sched:
                if mode == "poisson":
                    while time.perf_counter() - t0 < q.arrival:
                        pass
                start = time.perf_counter() - t0
                streams[q.stream_id](src(q.stream_id, q.frame))
                torch.cuda.synchronize()
                done = time.perf_counter() - t0
                results.append(serve.Result(q.stream_id, q.frame, q.arrival if mode == "poisson" else 0.0,
                                            start, done))
            out[f"plain_{mode}"] = serve.summarize(results, res)
            del streams
    out["clocks"] = clk.summary()
    out["chosen_vs_plain_saturated"] = round(out["chosen_saturated"]["frames_per_s"]
                                             / out["plain_saturated"]["frames_per_s"], 2)
    return out


def run_reference(a, device):
    H, W = a.height, a.width
    n = min(a.pool, a.warmup + a.steps)
    frames = make_frames(H, W, n, a.seed, device)
    band, alpha = fixed_prediction(H, W, a.seed, device)
    from oracle.reference_step import ReferenceStep
    cfg = stepmod.StepConfig(regression_width=a.win, filter_width=a.filter_win)
    mk = lambda: ReferenceStep(cfg.regression_width, cfg.sparsity, cfg.filter_width, cfg.win_curr, cfg.win_prev,
                               band, alpha)
    stream = torch.cuda.current_stream()
    rs = mk()
    with Clocks(device) as clk:
        total, ms = timed_steps(lambda f, t: rs(f), frames, a.warmup, a.steps, stream)
    res = {"value": a.steps / (total * 1e-3), "ms_per_step": total / a.steps, "p50_ms": pct(ms, 50),
           "p99_ms": pct(ms, 99), "clocks": clk.summary()}
    host = [{k: v.cpu().pin_memory() for k, v in frames[i].items()} for i in range(min(4, n))]
    dev_in = [{k: torch.empty_like(v) for k, v in frames[0].items()} for _ in range(2)]
    out_host = torch.empty((1, H, W, 3), dtype=torch.float32).pin_memory()
    rs2 = mk()

    def e2e_step(_f, t):
        slot = dev_in[t % 2]
        for k, v in host[t % len(host)].items():
            slot[k].copy_(v, non_blocking=True)
        o = rs2(slot)
        out_host.copy_(o["out"], non_blocking=True)

    e2e_steps = max(1, min(a.steps, 40))
    total, ms = timed_steps(e2e_step, frames, min(a.warmup, 4), e2e_steps, stream)
    h2d = sum(v.numel() * v.element_size() for v in host[0].values())
    res["e2e"] = {"value": e2e_steps / (total * 1e-3), "unit": "frames/s", "steps": e2e_steps,
                  "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(out_host.numel() * 4)}
    return res


def main():
    a = args_parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    config = {"workload": (f"{a.width}x{a.height} frame step of the hot path: log1p, cross_regression "
                           f"(win {a.win}, sparsity 4), Reproject of a 3-tensor history, 3x3 erosion + "
                           f"temporal screening (7/1), spatial filter (win {a.filter_win}) forward, aggregation "
                           f"loss forward/backward, spatial_filter_grad; band/alpha fixed (network step not "
                           f"included)"),
              "height": a.height, "width": a.width, "regression_win": a.win, "sparsity": 4,
              "filter_win": a.filter_win, "streams_per_gpu": 1,
              "l2": "inputs larger than L2: every step reads a new frame (182 MB of inputs)",
              "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}
    common = {"metric": METRIC, "unit": "frames/s", "n_gpus": world if a.impl == "mine" else 1,
              "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak",
              "vs_baseline": None, "dtype": "f32",
              "data": "synthetic: seeded Voronoi G-buffer sequence with camera pan and per-cell motion "
                      "(stands in for the reference's EXR scenes)",
              "config": config}

    if a.serve and a.impl == "mine":
        r = run_serving(a, device)
        print(json.dumps(dict(common, metric="aggregate denoised frames/sec and p50/p99 ms/frame, 16 mixed-"
                                             "resolution streams on 1 B200, chosen vs plain",
                              value=r["chosen_saturated"]["frames_per_s"], serving=r,
                              config=dict(config, workload="serving: 16 streams (4x1280x720, 8x1920x1080, "
                                                           "3x2560x1440, 1x3840x2160), Poisson 30-120 Hz, full "
                                                           "step with online U-Net training per frame"))))
        return

    if a.impl == "reference":
        if rank != 0:
            return
        from oracle import reference as ref
        if not ref.available():
            print(json.dumps({"impl": "reference",
                              "unavailable": "reference kernels not built (make -C oracle ref needs the "
                                             "reference sources)"}))
            return
        r = run_reference(a, device)
        line = dict(common, impl="reference", value=r["value"], ms_per_step=r["ms_per_step"],
                    p50_ms=r["p50_ms"], p99_ms=r["p99_ms"], e2e=r["e2e"], clocks=r["clocks"],
                    gpu_launches=None,
                    cpu_baseline={"kind": "reference", "device": "cuda", "cores": None, "value": r["value"],
                                  "unit": "frames/s",
                                  "sample": f"{a.steps} full frames on the reference's CUDA kernels"},
                    note=("the reference implements this path only as CUDA kernels; oracle/_ref holds them "
                          "compiled from the reference sources for sm_100a, driven as its TF op wrappers do"))
        print(json.dumps(line))
        return

    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=device)
    try:
        r = run_mine(a, rank, world, device)
        serving = None
        if world == 1 and not a.no_serve:
            # the 16-stream serving run (bounded: serve_frames per stream), on
            # a device emptied of the single-stream runs' buffers
            import gc
            gc.collect()
            torch.cuda.empty_cache()
            serving = run_serving(a, device)
        cpu = None
        if rank == 0 and world == 1 and not a.no_cpu_baseline:
            cpu = cpu_baseline(a.height, a.width, a.win, a.filter_win, a.seed)
        if rank == 0:
            line = dict(common, value=r["value"], ms_per_step=r["ms_per_step"], p50_ms=r["p50_ms"],
                        p99_ms=r["p99_ms"], plain=r["plain"], e2e=r["e2e"], gpu_launches=r["gpu_launches"],
                        roofline=r.get("roofline"), roofline_hbm=r.get("roofline_hbm"), cpu_baseline=cpu,
                        clocks=r["clocks"], per_op_ms=r["per_op_ms"],
                        sweep_frames_per_s=r.get("sweep_frames_per_s"), full_step=r.get("full_step"),
                        differentiation=r.get("differentiation"), serving=serving)
            print(json.dumps(line))
    finally:
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
