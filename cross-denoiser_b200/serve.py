"""Serving many camera streams of different resolutions on one GPU.

Each stream is a sequence of frames denoised by the reference's per-frame
train_step (scripts/main.py:250-313, history hand-off :323-341): the fused
ops plus its own online-trained U-Net.  Everything a stream carries from one
frame to the next (history buffers, network weights, Adam moments and step
count) stays resident in HBM for the life of the stream.

Scheduling (continuous batching): a request is one frame of one stream.
Frames of a stream run in order, one at a time (frame t+1 reads frame t's
history); frames of different streams run concurrently, each stream on its
own CUDA stream, so the work of requests that arrive while others are on the
GPU overlaps on the device.  A stream is admitted when its first request
arrives if its HBM footprint fits the budget next to the admitted streams;
otherwise it waits, and is admitted when finished streams release memory.

After its first frame (run eagerly, which allocates everything) a stream's
step is captured once as a CUDA graph for its resolution and replayed for
every later frame; the graph ends by copying the frame's outputs into the
stream's history buffers, so replays chain exactly like the eager step.
Inputs come either from device buffers (G-buffers rendered on the same GPU)
or from pinned host memory (copied in on the stream's CUDA stream).
"""
from __future__ import annotations

import gc
import time
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np
import torch

from . import step as stepmod
from . import synth
from .unet import UNet

# HBM bytes per pixel of one stream before it is measured (inputs slot,
# history, the step's intermediates, the U-Net workspace): an upper bound
# used for admission; the measured figure replaces it once a stream of that
# resolution has been built.
EST_BYTES_PER_PX = 1400


@dataclass
class Request:
    arrival: float          # seconds from the start of the run
    stream_id: int
    frame: int


@dataclass
class Result:
    stream_id: int
    frame: int
    arrival: float
    start: float
    done: float

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def poisson_schedule(rates_hz: List[float], frames: int, seed: int) -> List[Request]:
    """Per stream, `frames` arrivals with exponential gaps of mean 1 / rate."""
    rng = np.random.default_rng(seed)
    out = []
    for sid, r in enumerate(rates_hz):
        t = np.cumsum(rng.exponential(1.0 / r, size=frames))
        out += [Request(float(a), sid, i) for i, a in enumerate(t)]
    out.sort(key=lambda q: (q.arrival, q.stream_id))
    return out


class Session:
    """One camera stream's device-resident state and its per-frame step."""

    def __init__(self, sid: int, H: int, W: int, frame_source: Callable[[int], Dict[str, torch.Tensor]],
                 device, cfg: stepmod.StepConfig, seed: int, graphs: bool = True, keep_outputs: bool = False):
        self.sid, self.H, self.W = sid, H, W
        self.device = device
        self.source = frame_source
        self.cuda_stream = torch.cuda.Stream(device=device)
        self.net = UNet(device, seed=seed)
        self.step = stepmod.FrameStep(cfg, predictor=self.net, on_gradients=self.net.on_gradients)
        self.hist = stepmod.History.zeros(1, H, W, device)
        self.step.history = self.hist
        ex = frame_source(0)
        self.slot = {k: torch.empty_like(v, device=device) for k, v in ex.items()}
        self.out = torch.empty((1, H, W, 3), dtype=torch.float32, device=device)
        self.graphs = graphs
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self.next_frame = 0
        self.inflight: Optional[Tuple[Request, torch.cuda.Event, float]] = None
        self.keep_outputs = keep_outputs
        self.outputs: List[torch.Tensor] = []

    def _body(self):
        o = self.step(self.slot)
        h = self.hist
        h.out_log.copy_(o["out_log"])
        h.ols1.copy_(o["ols1"])
        h.ols2.copy_(o["ols2"])
        h.linearZ.copy_(self.slot["linearZ"])
        h.normal.copy_(self.slot["normal"])
        self.step.history = h
        self.out.copy_(o["out"])

    def launch(self, frame: int, host: Optional[Dict[str, torch.Tensor]] = None) -> torch.cuda.Event:
        """Enqueue one frame on this stream's CUDA stream; returns its done event."""
        with torch.cuda.stream(self.cuda_stream):
            src = host if host is not None else self.source(frame)
            for k, v in src.items():
                self.slot[k].copy_(v, non_blocking=True)
            if self.graph is not None:
                self.graph.replay()
            elif self.graphs and frame > 0:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=self.cuda_stream):
                    self._body()
                self.graph = g
                g.replay()
            else:
                self._body()
            if self.keep_outputs:
                self.outputs.append(self.out.clone())
            self.net.enqueue_error_readback()
            ev = torch.cuda.Event()
            ev.record(self.cuda_stream)
        self.next_frame = frame + 1
        return ev

    def check(self):
        """Raise if this stream's network reported a tensor-core time-out in
        a frame whose done event has completed."""
        self.net.raise_if_failed()

    def release(self):
        """Free the device state (outputs kept with keep_outputs survive)."""
        self.graph = None
        self.net = None
        self.step = None
        self.slot = self.out = self.hist = None


class Server:
    """Continuous-batching request loop over sessions (see module docstring).

    `session_factory(sid, H, W, source)` builds a stream's state (Session by
    default) and `memory_probe()` reports allocated device bytes; both are
    parameters so the scheduling logic can run against stand-ins.
    """

    def __init__(self, resolutions: List[Tuple[int, int]], frame_source, device, hbm_budget: int,
                 cfg: Optional[stepmod.StepConfig] = None, graphs: bool = True, seed: int = 0,
                 keep_outputs: bool = False, session_factory=None, memory_probe=None):
        self.res = resolutions
        self.source = frame_source                  # (sid, frame) -> dict of device tensors
        self.device = device
        self.budget = int(hbm_budget)
        self.cfg = cfg or stepmod.StepConfig(fused=True)
        self.seed = seed
        self.factory = session_factory or (lambda sid, H, W, src: Session(
            sid, H, W, src, device, self.cfg, seed=self.seed + sid, graphs=graphs, keep_outputs=keep_outputs))
        self.memory = memory_probe or (lambda: torch.cuda.memory_allocated(device))
        self.sessions: Dict[int, "Session"] = {}
        self.retired: Dict[int, "Session"] = {}
        self.footprint: Dict[int, int] = {}
        self.measured: Dict[Tuple[int, int], int] = {}
        self.max_admitted = 0
        self.admission_waits = 0

    def calibrate(self, frames: int = 2):
        """Build one stream per distinct resolution, run `frames` frames
        (eager first frame, graph capture, replay), record its device
        footprint for admission and release it."""
        for (H, W) in sorted(set(self.res)):
            sid = self.res.index((H, W))
            gc.collect()
            torch.cuda.synchronize(self.device)
            before = self.memory()
            s = self.factory(sid, H, W, lambda t, sid=sid: self.source(sid, t))
            for t in range(frames):
                s.launch(t)
            torch.cuda.synchronize(self.device)
            self.measured[(H, W)] = self.memory() - before
            s.release()
            del s
        gc.collect()
        torch.cuda.synchronize(self.device)

    def admit_all(self) -> int:
        """Admit every stream that fits the budget now, in stream order;
        returns how many are resident."""
        for sid in range(len(self.res)):
            if sid not in self.sessions and sid not in self.retired and not self._admit(sid):
                break
        return len(self.sessions)

    def warm(self, frames: int = 2):
        """Run the first `frames` frames of every resident stream (the eager
        first frame that allocates the stream's buffers, the graph capture)
        outside any timed region; run() then continues from frame `frames`."""
        for s in self.sessions.values():
            for t in range(frames):
                s.launch(t)
        if torch.cuda.is_available():
            torch.cuda.synchronize(self.device)

    def _estimate(self, sid):
        H, W = self.res[sid]
        return self.measured.get((H, W), EST_BYTES_PER_PX * H * W)

    def _admit(self, sid) -> bool:
        need = self._estimate(sid)
        if sum(self.footprint.values()) + need > self.budget:
            return False
        H, W = self.res[sid]
        self.sessions[sid] = self.factory(sid, H, W, lambda t, sid=sid: self.source(sid, t))
        self.footprint[sid] = need
        self.max_admitted = max(self.max_admitted, len(self.sessions))
        return True

    def _retire(self, sid):
        s = self.sessions.pop(sid)
        self.footprint.pop(sid)
        self.retired[sid] = s
        s.release()

    def run(self, schedule: List[Request], frames_per_stream: int, realtime: bool = True) -> List[Result]:
        """Serve the schedule; with realtime False every request is ready at
        once (saturation throughput)."""
        pending: Dict[int, List[Request]] = {}
        for q in schedule:
            pending.setdefault(q.stream_id, []).append(q)
        waiting = sorted((sid for sid in pending if sid not in self.sessions),
                         key=lambda sid: pending[sid][0].arrival)
        results: List[Result] = []
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        total = len(schedule)
        while len(results) < total:
            t = now()
            # completions
            for sid, s in list(self.sessions.items()):
                if s.inflight is not None and s.inflight[1].query():
                    q, _, start = s.inflight
                    if hasattr(s, "check"):
                        s.check()
                    results.append(Result(sid, q.frame, q.arrival if realtime else 0.0, start, now()))
                    s.inflight = None
                    if s.next_frame >= frames_per_stream:
                        self._retire(sid)
            # admissions, in order of first arrival; a stream that does not fit
            # waits (and so do the ones behind it) until memory is released
            while waiting and (not realtime or pending[waiting[0]][0].arrival <= t):
                if not self._admit(waiting[0]):
                    self.admission_waits += 1
                    if not self.sessions:
                        raise MemoryError(f"stream {waiting[0]} does not fit the HBM budget on its own")
                    break
                waiting.pop(0)
            # dispatch: every admitted stream whose next frame has arrived and
            # that has nothing in flight
            for sid, s in self.sessions.items():
                if s.inflight is None and pending[sid] and (not realtime or pending[sid][0].arrival <= t):
                    q = pending[sid].pop(0)
                    start = now()
                    s.inflight = (q, s.launch(q.frame), start)
        if torch.cuda.is_available():
            torch.cuda.synchronize(self.device)
        return results


def summarize(results: List[Result], resolutions) -> dict:
    """Throughput over the span of the results, latency from arrival to the
    denoised frame (queueing included) and service time from dispatch to the
    denoised frame, overall and per resolution."""
    lat = np.array([r.latency for r in results]) * 1e3
    svc = np.array([r.done - r.start for r in results]) * 1e3
    span = max(r.done for r in results) - min(min(r.start for r in results), min(r.arrival for r in results))
    by_res = {}
    for (H, W) in sorted(set(resolutions)):
        ls = np.array([r.latency for r in results if resolutions[r.stream_id] == (H, W)]) * 1e3
        ss = np.array([r.done - r.start for r in results if resolutions[r.stream_id] == (H, W)]) * 1e3
        by_res[f"{W}x{H}"] = {"frames": int(ls.size), "p50_ms": round(float(np.percentile(ls, 50)), 3),
                              "p99_ms": round(float(np.percentile(ls, 99)), 3),
                              "service_p50_ms": round(float(np.percentile(ss, 50)), 3),
                              "service_p99_ms": round(float(np.percentile(ss, 99)), 3)}
    px = sum(resolutions[r.stream_id][0] * resolutions[r.stream_id][1] for r in results)
    return {"frames": len(results), "seconds": round(span, 3), "frames_per_s": round(len(results) / span, 2),
            "megapixels_per_s": round(px / span / 1e6, 1),
            "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "service_p50_ms": round(float(np.percentile(svc, 50)), 3),
            "service_p99_ms": round(float(np.percentile(svc, 99)), 3), "by_resolution": by_res}


def device_frame_source(resolutions, seeds, device, pool: int = 4):
    """A small pool of distinct frames per stream, generated on the device and
    cycled (frame t of stream s is pool entry t % pool of its own sequence)."""
    cache = {}

    def src(sid, t):
        if sid not in cache:
            H, W = resolutions[sid]
            seq = synth.make_sequence(H, W, seed=seeds[sid], object_motion=4.0, device=device,
                                      max_frames=pool + 2)
            cache[sid] = [{k: v for k, v in seq.frame(i).items() if k in synth.FRAME_INPUTS}
                          for i in range(pool)]
        return cache[sid][t % len(cache[sid])]
    return src
