"""Per-frame step of the online denoiser on the sm_100a ops.

Mirrors the op order of the reference's train_step (scripts/main.py:250-313):

  1. y1, y2 = log1p(color), log1p(color2)                        (:207-212)
  2. ols1, ols2, var1, var2 = cross_regression(y1, y2, albedo, normal)  (:261)
  3. success, [prev out_log, ols1, ols2] = Reproject(...)         (:266)
     with opacity and previous opacity both all-ones, as the reference passes
  4. 3x3 erosion of float(success)                                (:270-276)
  5. prev_out, prev_ols1, prev_ols2, success_prev = temporal_screening(...,
     win_curr=7, win_prev=1)                                      (:280)
  6. band, alpha = predictor(ols1, ols2, prev_out, albedo, normal) (:291)
  7. sum1, sum2, sumw1, sumw2 = spatial_filter(ols1, ols2, albedo, normal,
     band, win_size=11)                                           (:295)
  8. aggregation loss with labels crossed (label1 = ols2, ...)    (:214-248, 283-286)
  9. dL/dband through spatial_filter_grad; dL/dalpha              (:302)
 10. history hand-off: out_log, ols1, ols2, linearZ, normal       (:338-341)

The predictor (the reference's kernel-predicting U-Net and its Adam update)
is pluggable: ``FrameStep(predictor=...)`` takes any callable returning
(band [B,H,W,5], alpha [B,H,W,1]) and receives the gradients through
``on_gradients``; by default a fixed band/alpha is used.

``plain`` runs the drop-in op sequence (separate erosion, screening,
filter, aggregation and gradient kernels); ``fused`` runs erosion with
screening as one kernel and the filter, aggregation loss and band gradient
as one kernel.  The two agree within rounding of the loss terms; the masks,
the filtered frame and the history are identical.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, Optional

import torch

from . import ops

REGRESSION_WIDTH = 17      # scripts/main.py:71
FILTER_WIDTH = 11          # scripts/main.py:72
SPARSITY = 4               # scripts/main.py:73
WIN_CURR, WIN_PREV = 7, 1  # scripts/main.py:280


@dataclass
class StepConfig:
    regression_width: int = REGRESSION_WIDTH
    filter_width: int = FILTER_WIDTH
    sparsity: int = SPARSITY
    win_curr: int = WIN_CURR
    win_prev: int = WIN_PREV
    fused: bool = False
    # > 0: re-solve ill-conditioned regression centres in FP64 (condition
    # estimate above this value); the count per frame is returned as
    # "fp64_fallbacks".  0 keeps the reference's FP32 solve.
    fp64_cond_limit: float = 0.0
    # True: the predictor's training update (on_gradients: the U-Net
    # backward and Adam) runs on a training stream of its own, overlapping
    # the next frame's regression, reprojection and screening; the next
    # prediction waits for it.  Same results as the serial order.
    overlap_training: bool = False


@dataclass
class History:
    """Per-stream state carried from one frame to the next
    (scripts/main.py:323-341); zeros before the first frame."""
    out_log: torch.Tensor
    ols1: torch.Tensor
    ols2: torch.Tensor
    linearZ: torch.Tensor
    normal: torch.Tensor

    @staticmethod
    def zeros(B, H, W, device) -> "History":
        z = lambda: torch.zeros((B, H, W, 3), dtype=torch.float32, device=device)
        return History(z(), z(), z(), z(), z())


class FrameStep:
    """One stream's per-frame denoise + loss + gradient step."""

    def __init__(self, cfg: StepConfig = StepConfig(), predictor: Optional[Callable] = None,
                 on_gradients: Optional[Callable] = None):
        self.cfg = cfg
        self.predictor = predictor
        self.on_gradients = on_gradients
        self.history: Optional[History] = None
        self._ones: Optional[torch.Tensor] = None
        self.fixed_band: Optional[torch.Tensor] = None
        self.fixed_alpha: Optional[torch.Tensor] = None
        self._train_stream: Optional[torch.cuda.Stream] = None
        self._trained: Optional[torch.cuda.Event] = None
        self._held = None   # gradients the training stream may still be reading
        self._side: Optional[torch.cuda.Stream] = None   # reprojection beside the regression

    def reset(self):
        self.history = None

    def wait_training(self, stream: Optional[torch.cuda.Stream] = None):
        """Make `stream` (default: the current one) wait for the last training
        update enqueued with overlap_training; call it before reading the
        predictor's parameters."""
        if self._trained is not None:
            st = stream or torch.cuda.current_stream()
            st.wait_event(self._trained)
            if st == torch.cuda.current_stream():
                # later allocations on this stream are ordered after the update,
                # so the gradients' memory may be reused from here on
                self._held = None

    def _train(self, g_band, g_alpha, device):
        if not self.cfg.overlap_training:
            self.on_gradients(g_band, g_alpha)
            return
        if self._train_stream is None:
            # high priority: the update's small, latency-bound kernels are
            # placed first and the next frame's FP32-bound ops fill the SMs
            self._train_stream = torch.cuda.Stream(device, priority=-1)
            self._trained = torch.cuda.Event()
        ts = self._train_stream
        ts.wait_stream(torch.cuda.current_stream(device))
        with torch.cuda.stream(ts):
            self.on_gradients(g_band, g_alpha)
        self._trained.record(ts)
        # the gradients were allocated on the compute stream: keep them alive
        # until that stream has waited for this update (next prediction)
        self._held = (g_band, g_alpha)

    def set_fixed_prediction(self, band: torch.Tensor, alpha: torch.Tensor):
        self.fixed_band, self.fixed_alpha = band, alpha

    def __call__(self, f: Dict[str, torch.Tensor]) -> Dict[str, torch.Tensor]:
        cfg = self.cfg
        color = f["color"]
        B, H, W, _ = color.shape
        if self.history is None:
            self.history = History.zeros(B, H, W, color.device)
        h = self.history
        albedo, normal = f["albedo"], f["normal"]

        # the reference reprojects with opacity 1 everywhere (scripts/main.py:266):
        # one constant tensor per shape, not a fill per frame
        if self._ones is None or self._ones.shape != (B, H, W, 1) or self._ones.device != color.device:
            self._ones = torch.ones((B, H, W, 1), dtype=torch.float32, device=color.device)
        ones1 = self._ones

        def reproject():
            return ops.Reproject(f["mvec"], [h.out_log, h.ols1, h.ols2], f["linearZ"], h.linearZ, normal,
                                 h.normal, f["pnFwidth"], ones1, ones1)

        compute = torch.cuda.current_stream(color.device)
        if cfg.fused:
            # reprojection (bandwidth-bound) needs only the history and this
            # frame's G-buffer: run it on a side stream beside the (FP32-bound)
            # regression.  The side stream first waits for all earlier work
            # here, so memory it reuses is no longer read.
            if self._side is None:
                self._side = torch.cuda.Stream(color.device)
            self._side.wait_stream(compute)
            with torch.cuda.stream(self._side):
                success, rep = reproject()
        y1, y2 = ops.prepare_input(color, f["color2"])
        fallbacks = None
        if cfg.fp64_cond_limit > 0:
            fallbacks = torch.zeros((1,), dtype=torch.int32, device=color.device)
        ols1, ols2, _, _ = ops.cross_regression(y1, y2, albedo, normal, win_size=cfg.regression_width,
                                                sparsity=cfg.sparsity, fp64_cond_limit=cfg.fp64_cond_limit,
                                                fallback_count=fallbacks)
        if cfg.fused:
            compute.wait_stream(self._side)
        else:
            success, rep = reproject()
        if cfg.fused:
            prev_out, prev_ols1, prev_ols2, success_prev, success_f = ops.erode_temporal_screening(
                ols1, ols2, rep[0], rep[1], rep[2], success, cfg.win_curr, cfg.win_prev)
        else:
            success_f = ops.erode3x3(success)
            prev_out, prev_ols1, prev_ols2, success_prev = ops.temporal_screening(
                ols1, ols2, rep[0], rep[1], rep[2], success_f, win_curr=cfg.win_curr, win_prev=cfg.win_prev)
        if self.predictor is not None:
            self.wait_training()
            band, alpha = self.predictor(ols1, ols2, prev_out, albedo, normal)
        else:
            band, alpha = self.fixed_band, self.fixed_alpha
        band, alpha = band.detach(), alpha.detach()
        loss = None
        if cfg.fused:
            out_log, out, avg, g_band, g_alpha = ops.filter_aggregate(
                ols1, ols2, albedo, normal, band, alpha, success_f, success_prev, prev_out, f["opacity"],
                prev_ols1, prev_ols2, win_size=cfg.filter_width)
        else:
            sum1, sum2, sumw1, sumw2 = ops.spatial_filter(ols1, ols2, albedo, normal, band,
                                                          win_size=cfg.filter_width)
            (out_log, out, loss, avg, g1, gw1, g2, gw2, g_alpha) = ops.aggregation_loss(
                sum1, sumw1, sum2, sumw2, alpha, success_f, success_prev, prev_out, f["opacity"],
                ols2, ols1, prev_ols2, prev_ols1)
            g_band = ops.spatial_filter_grad(g1, g2, gw1, gw2, ols1, ols2, albedo, normal, band,
                                             win_size=cfg.filter_width)
        if self.on_gradients is not None:
            self._train(g_band, g_alpha, color.device)
        self.history = History(out_log, ols1, ols2, f["linearZ"], normal)
        return {"out": out, "out_log": out_log, "loss": loss, "avg_loss": avg, "ols1": ols1, "ols2": ols2,
                "g_band": g_band, "g_alpha": g_alpha, "success": success, "band": band, "alpha": alpha,
                "fp64_fallbacks": fallbacks}


class HostFramePipeline:
    """Denoises frames held in host memory with the copies off the critical path.

    ``pipe(host_frame)`` enqueues frame t: its inputs are copied to the device
    on an upload stream, the step runs on the caller's current stream, and the
    denoised frame (and the average loss) are read back on a download stream.
    PCIe is full duplex and the copy engines run beside the SMs, so frame t+1
    uploads and frame t-1 downloads while frame t computes; the frame rate is
    bound by the slower of the upload and the step instead of their sum.

    Frames of one stream keep their order: frame t+1 reads frame t's history,
    and its linearZ and normal stay in frame t's input slot, so three slots
    rotate (the slot of frame t+1 is free once frame t has finished reading
    frame t-1's history).  Returns (out, avg_loss, event): pinned host tensors
    that hold the result once ``event`` has completed, valid until the call
    two frames later reuses them.  Host frames should be pinned for the
    copies to be asynchronous.
    """

    SLOTS = 3

    def __init__(self, step: FrameStep, device=None):
        self.step = step
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.up = torch.cuda.Stream(self.device)
        self.down = torch.cuda.Stream(self.device)
        self.slots = None
        self.t = 0
        self.released = [torch.cuda.Event() for _ in range(self.SLOTS)]
        self.uploaded = [torch.cuda.Event() for _ in range(self.SLOTS)]
        self.computed = torch.cuda.Event()
        self.read_back = [torch.cuda.Event() for _ in range(2)]
        self.out_host = None
        self.loss_host = None
        self.pending = [None, None]   # device results being read back

    def _alloc(self, host_frame):
        self.slots = [{k: torch.empty(v.shape, dtype=v.dtype, device=self.device) for k, v in host_frame.items()}
                      for _ in range(self.SLOTS)]
        B, H, W, _ = host_frame["color"].shape
        self.out_host = [torch.empty((B, H, W, 3), dtype=torch.float32).pin_memory() for _ in range(2)]
        self.loss_host = [torch.empty((), dtype=torch.float32).pin_memory() for _ in range(2)]

    def __call__(self, host_frame: Dict[str, torch.Tensor]):
        if self.slots is None:
            self._alloc(host_frame)
        t, s, o = self.t, self.t % self.SLOTS, self.t % 2
        compute = torch.cuda.current_stream(self.device)
        if self.pending[o] is not None:
            # frame t-2's results were allocated on the compute stream and read
            # on the download stream: order later allocations after that read
            compute.wait_event(self.read_back[o])
            self.pending[o] = None
        # slot s last held frame t-3, which frame t-2 read as history
        if t >= self.SLOTS:
            self.up.wait_event(self.released[s])
        with torch.cuda.stream(self.up):
            for k, v in host_frame.items():
                self.slots[s][k].copy_(v, non_blocking=True)
            self.uploaded[s].record(self.up)
        compute.wait_event(self.uploaded[s])
        r = self.step(self.slots[s])
        if t >= 1:
            # frame t has read frame t-1's linearZ/normal (its history)
            self.released[(t - 1) % self.SLOTS].record(compute)
        self.computed.record(compute)
        # the host buffers of frame t-2 must have been read back before reuse
        self.down.wait_event(self.computed)
        with torch.cuda.stream(self.down):
            self.out_host[o].copy_(r["out"], non_blocking=True)
            self.loss_host[o].copy_(r["avg_loss"], non_blocking=True)
            self.read_back[o].record(self.down)
        self.pending[o] = (r["out"], r["avg_loss"])
        self.t += 1
        return self.out_host[o], self.loss_host[o], self.read_back[o]

    def drain(self, stream=None):
        """Make `stream` (default: the current one) wait for every enqueued copy."""
        st = stream or torch.cuda.current_stream(self.device)
        st.wait_stream(self.up)
        st.wait_stream(self.down)
