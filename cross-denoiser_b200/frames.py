"""Frame sequences on disk: the reference's NPY scene layout.

The reference reads a scene directory of one file per buffer and frame,
``{type}_{frame:04d}.exr``, converts every EXR once to ``.npy`` next to it
(``[1, H, W, C]`` float32, NaN and +-Inf set to zero) and then loads the NPY
files frame by frame (scripts/utils.py:49-70 load_exr / save_as_npy,
:147-305 DataLoader; buffer list scripts/main.py:60-65).  ``NpySequence``
reads that NPY layout with the same validation (every type present, the
same frame indices for every type, frames below ``max_num_frames``) and the
same indexing (item i is frame start + i % num_frames, ``skip_frames``),
and hands frames out as pinned host tensors for ``step.HostFramePipeline``,
optionally read ahead on a background thread.  EXR decoding is not built
(OpenEXR is not available here): ``.exr``-only directories are refused with
that reason, and NPY files written by the reference's conversion (or by
``save_npy_sequence``) are read as they are.

Also the two per-frame steps of the reference's driver around the denoiser:
``compose_output`` adds the emissive and environment-light buffers to the
denoised frame (scripts/main.py:345) and ``rel_l2`` is its error metric
(scripts/main.py:191-197).
"""
from __future__ import annotations

import os
import queue
import re
import threading
from typing import Dict, Iterable, List, Optional, Tuple

import numpy as np
import torch

# buffers the reference's driver reads (scripts/main.py:60-65)
READ_TYPES = ("ref", "color", "color2", "albedo", "normal", "mvec", "linearZ", "pnFwidth", "opacity",
              "emissive", "envLight", "ref_emissive", "ref_envLight")
# the subset the denoiser's per-frame step consumes
STEP_TYPES = ("color", "color2", "albedo", "normal", "mvec", "linearZ", "pnFwidth", "opacity")

_NAME = re.compile(r"^(?P<type>.+)_(?P<frame>\d+)\.(?P<ext>npy|exr)$")


def _scan(directory: str, types: Iterable[str], max_num_frames: Optional[int]) -> Dict[str, Dict[int, str]]:
    """type -> {frame: path} of the files named {type}_{frame}.npy|exr."""
    types = set(types)
    found: Dict[str, Dict[int, str]] = {}
    exr_only: Dict[str, Dict[int, str]] = {}
    for name in sorted(os.listdir(directory)):
        m = _NAME.match(name)
        if not m or m.group("type") not in types:
            continue
        frame = int(m.group("frame"))
        if max_num_frames is not None and frame >= max_num_frames:
            continue
        dst = found if m.group("ext") == "npy" else exr_only
        dst.setdefault(m.group("type"), {})[frame] = os.path.join(directory, name)
    if not found and exr_only:
        raise RuntimeError(f"{directory}: only .exr files; EXR decoding is not available in this build, "
                           "convert the scene to .npy ([1,H,W,C] float32 per file) first")
    if not found:
        raise FileNotFoundError(f"{directory}: no {{type}}_{{frame:04d}}.npy files of types {sorted(types)}")
    missing = types - set(found)
    if missing:
        raise ValueError(f"{directory}: types {sorted(missing)} are not given")
    counts = {t: len(f) for t, f in found.items()}
    if len(set(counts.values())) != 1:
        raise ValueError(f"{directory}: different number of files per type: {counts}")
    ref_frames = None
    for t, f in sorted(found.items()):
        if ref_frames is None:
            ref_frames = set(f)
        elif set(f) != ref_frames:
            raise ValueError(f"{directory}: {t} has different frame indices than the other types")
    return found


def load_npy(path: str) -> np.ndarray:
    """One buffer as [1, H, W, C] float32 with NaN and +-Inf set to zero (the
    reference's save_as_npy sanitisation, scripts/utils.py:58-66)."""
    a = np.load(path)
    if a.ndim == 3:
        a = a[None]
    if a.ndim != 4 or a.shape[0] != 1:
        raise ValueError(f"{path}: expected [1,H,W,C], got {a.shape}")
    a = np.ascontiguousarray(a, dtype=np.float32)
    if not np.isfinite(a).all():
        a = np.nan_to_num(a, nan=0.0, posinf=0.0, neginf=0.0)
    return a


class NpySequence:
    """A scene directory of {type}_{frame:04d}.npy files (see module docstring).

    ``seq[i]`` returns (frame index, {type: pinned [1,H,W,C] float32 tensor});
    ``frame(t)`` the buffers of absolute frame t.
    """

    def __init__(self, directory: str, types: Iterable[str] = STEP_TYPES, max_num_frames: Optional[int] = 101,
                 pin: bool = True):
        self.directory = directory
        self.types = tuple(types)
        self.files = _scan(directory, self.types, max_num_frames)
        frames = sorted(next(iter(self.files.values())))
        self.start_frame = frames[0]
        self.num_frames = len(frames)
        self.frames = frames
        self.pin = pin and torch.cuda.is_available()

    def skip_frames(self, n: int):
        """Drop the first n frames (scripts/utils.py:264-266)."""
        self.start_frame += n
        self.num_frames -= n
        self.frames = self.frames[n:]

    def __len__(self) -> int:
        return self.num_frames

    def frame(self, t: int) -> Dict[str, torch.Tensor]:
        out = {}
        for typ in self.types:
            path = self.files[typ].get(t)
            if path is None:
                raise KeyError(f"frame {t} of {typ} is not in {self.directory}")
            x = torch.from_numpy(load_npy(path))
            out[typ] = x.pin_memory() if self.pin else x
        shapes = {tuple(v.shape[:3]) for v in out.values()}
        if len(shapes) != 1:
            raise ValueError(f"frame {t}: buffers differ in size: {shapes}")
        return out

    def __getitem__(self, index: int) -> Tuple[int, Dict[str, torch.Tensor]]:
        # the reference wraps the item index over the sequence (scripts/utils.py:288-290)
        t = self.frames[index % self.num_frames]
        return t, self.frame(t)

    def __iter__(self):
        for i in range(self.num_frames):
            yield self[i]

    def prefetch(self, depth: int = 2):
        """Iterate the sequence with the next `depth` frames read on a
        background thread (file reads overlap the GPU step)."""
        q: "queue.Queue" = queue.Queue(maxsize=max(1, depth))
        stop = object()

        def work():
            try:
                for item in self:
                    q.put(item)
            except BaseException as e:   # re-raised in the consumer
                q.put(e)
            q.put(stop)

        th = threading.Thread(target=work, daemon=True)
        th.start()
        while True:
            item = q.get()
            if item is stop:
                break
            if isinstance(item, BaseException):
                raise item
            yield item
        th.join()


def save_npy_sequence(directory: str, frames: List[Dict[str, torch.Tensor]], start: int = 0):
    """Write frames as {type}_{frame:04d}.npy, [1,H,W,C] float32 (the layout
    NpySequence reads)."""
    os.makedirs(directory, exist_ok=True)
    for i, f in enumerate(frames):
        for typ, v in f.items():
            a = v.detach().cpu().numpy().astype(np.float32)
            if a.ndim == 3:
                a = a[None]
            np.save(os.path.join(directory, f"{typ}_{start + i:04d}.npy"), a)


def compose_output(out: torch.Tensor, emissive: torch.Tensor, env_light: torch.Tensor) -> torch.Tensor:
    """The displayed frame: denoised radiance plus the emissive and
    environment-light buffers, which bypass the denoiser (scripts/main.py:345)."""
    return out + emissive + env_light


def rel_l2(pred, true):
    """Per-element relative squared error of the reference's driver
    (scripts/main.py:191-197): (true - pred)^2 / (mean_c(true)^2 + 1e-2);
    the printed figure is its mean."""
    true_mean = true.mean(-1, keepdim=True) if isinstance(true, torch.Tensor) else np.mean(true, -1, keepdims=True)
    return (true - pred) ** 2 / (true_mean ** 2 + 1e-2)
