"""Seeded synthetic frame sequences with the reference's G-buffer layout.

The reference evaluates on its own EXR dataset (read by scripts/utils.py's
DataLoader, buffers listed in scripts/main.py:60-65), which is not available
here.  This generator produces the same buffer set, channel counts and value
ranges so that every code path of the hot path is exercised:

* a Voronoi scene (64 cells by default) in world coordinates; each cell has
  a U(0.05, 0.95) albedo, a tilted plane (depth in [1, 50], constant unit
  normal) and optionally its own motion (+-object_motion px/frame);
* a camera panning 0.5-3 px/frame in a fixed direction with +-0.25 px jitter;
* color / color2: two independent half-sample-count radiance estimates,
  albedo x shading x lognormal(mu=-1, sigma=1.5) noise, with 0.1 % fireflies
  scaled by 100;
* linearZ = (depth, fwidth(depth), 0); pnFwidth = (fwidth(depth),
  fwidth(normal), 0); mvec = screen motion to the previous frame divided by
  (W, H), so prev = pos + mvec * dim (ops/reproject.cu.cc:97,103); opacity = 1;
  emissive / envLight: sparse (2 %) HDR values.

All tensors are NHWC float32 [1,H,W,C] on the requested device.  The same
(seed, frame, device) always gives the same frame.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Dict

import torch

BUFFERS = {"color": 3, "color2": 3, "albedo": 3, "normal": 3, "mvec": 3, "linearZ": 3,
           "pnFwidth": 3, "opacity": 1, "emissive": 3, "envLight": 3}

# the reproject / regression inputs that travel host -> device every frame
FRAME_INPUTS = ("color", "color2", "albedo", "normal", "mvec", "linearZ", "pnFwidth", "opacity")


@dataclass
class SceneSpec:
    H: int
    W: int
    seed: int = 0
    n_cells: int = 64
    object_motion: float = 0.0      # max per-cell motion in px/frame
    firefly_frac: float = 1e-3
    firefly_gain: float = 100.0
    emissive_frac: float = 0.02
    max_frames: int = 512


class SyntheticSequence:
    """Deterministic frame sequence; ``frame(t)`` renders frame t."""

    def __init__(self, spec: SceneSpec, device="cpu"):
        self.spec = spec
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(1000003 * spec.seed + 17)
        H, W, K = spec.H, spec.W, spec.n_cells
        ang = float(torch.rand((), generator=g)) * 2 * math.pi
        speed = 0.5 + 2.5 * float(torch.rand((), generator=g))
        jitter = (torch.rand((spec.max_frames, 2), generator=g) - 0.5) * 0.5
        pan = torch.tensor([math.cos(ang), math.sin(ang)]) * speed + jitter      # px / frame
        pan[0] = 0.0
        self.pan = pan
        self.cam = torch.cumsum(pan, 0)                                          # camera offset
        span = float(self.cam.abs().max()) + 4.0 * spec.object_motion * spec.max_frames ** 0.5 + 8
        lo = torch.tensor([-span, -span])
        hi = torch.tensor([W + span, H + span])
        area = float((hi - lo).prod())
        # keep the cell density of n_cells over the visible frame
        n = max(K, int(K * area / (H * W)))
        self.seeds = lo + torch.rand((n, 2), generator=g) * (hi - lo)
        self.vel = (torch.rand((n, 2), generator=g) * 2 - 1) * spec.object_motion
        self.albedo = 0.05 + 0.9 * torch.rand((n, 3), generator=g)
        tilt = (torch.rand((n, 2), generator=g) * 2 - 1) * 0.05                 # depth slope
        self.z0 = 1.0 + 49.0 * torch.rand((n,), generator=g)
        self.grad = tilt
        nz = torch.ones((n, 1))
        nrm = torch.cat([-tilt * 8.0, nz], 1)
        self.normal = nrm / nrm.norm(dim=1, keepdim=True)
        light = torch.tensor([0.3, 0.5, 0.81])
        self.shade = (self.normal @ (light / light.norm())).clamp(0.1, 1.0)
        for name in ("seeds", "vel", "albedo", "z0", "grad", "normal", "shade", "pan", "cam"):
            setattr(self, name, getattr(self, name).to(self.device))

    def _cells(self, t: int):
        H, W = self.spec.H, self.spec.W
        dev = self.device
        ys, xs = torch.meshgrid(torch.arange(H, device=dev, dtype=torch.float32),
                                torch.arange(W, device=dev, dtype=torch.float32), indexing="ij")
        wx = (xs + self.cam[t, 0]).reshape(-1)
        wy = (ys + self.cam[t, 1]).reshape(-1)
        sx = self.seeds[:, 0] + self.vel[:, 0] * t
        sy = self.seeds[:, 1] + self.vel[:, 1] * t
        idx = torch.empty(H * W, dtype=torch.long, device=dev)
        chunk = 1 << 18
        for s in range(0, H * W, chunk):
            d = (wx[s:s + chunk, None] - sx[None]) ** 2 + (wy[s:s + chunk, None] - sy[None]) ** 2
            idx[s:s + chunk] = d.argmin(1)
        rel_x = wx - sx[idx]
        rel_y = wy - sy[idx]
        return idx, rel_x, rel_y

    @staticmethod
    def _fwidth(img: torch.Tensor) -> torch.Tensor:
        # |d/dx| + |d/dy| with forward differences (edge replicated), summed over channels
        dx = torch.zeros_like(img)
        dy = torch.zeros_like(img)
        dx[:, :-1] = (img[:, 1:] - img[:, :-1]).abs()
        dx[:, -1] = dx[:, -2] if img.shape[1] > 1 else 0
        dy[:-1] = (img[1:] - img[:-1]).abs()
        dy[-1] = dy[-2] if img.shape[0] > 1 else 0
        return (dx + dy).sum(-1)

    def frame(self, t: int) -> Dict[str, torch.Tensor]:
        spec = self.spec
        H, W = spec.H, spec.W
        dev = self.device
        idx, rx, ry = self._cells(t)
        albedo = self.albedo[idx].reshape(H, W, 3)
        normal = self.normal[idx].reshape(H, W, 3)
        depth = (self.z0[idx] + self.grad[idx, 0] * rx + self.grad[idx, 1] * ry).clamp(1.0, 50.0)
        depth = depth.reshape(H, W, 1)
        fz = self._fwidth(depth)
        fn = self._fwidth(normal)
        zero = torch.zeros((H, W), device=dev)
        linz = torch.stack([depth[..., 0], fz, zero], -1)
        pnfw = torch.stack([fz, fn, zero], -1)
        motion = self.pan[t][None] - self.vel[idx]                  # px to the previous frame
        mvec = torch.stack([motion[:, 0] / W, motion[:, 1] / H, torch.zeros_like(motion[:, 0])], -1)
        mvec = mvec.reshape(H, W, 3)
        g = torch.Generator(device=dev).manual_seed(7919 * spec.seed + 104729 * t + 1)
        radiance = (albedo * self.shade[idx].reshape(H, W, 1) * 2.0)

        def noisy():
            n = torch.exp(torch.randn((H, W, 3), generator=g, device=dev) * 1.5 - 1.0)
            c = radiance * n
            ff = torch.rand((H, W, 1), generator=g, device=dev) < spec.firefly_frac
            return torch.where(ff, c * spec.firefly_gain, c)

        color = noisy()
        color2 = noisy()

        def sparse_hdr():
            m = torch.rand((H, W, 1), generator=g, device=dev) < spec.emissive_frac
            v = torch.exp(torch.randn((H, W, 3), generator=g, device=dev) + 1.0)
            return torch.where(m, v, torch.zeros_like(v))

        out = {
            "color": color, "color2": color2, "albedo": albedo, "normal": normal,
            "mvec": mvec, "linearZ": linz, "pnFwidth": pnfw,
            "opacity": torch.ones((H, W, 1), device=dev),
            "emissive": sparse_hdr(), "envLight": sparse_hdr(),
        }
        return {k: v.unsqueeze(0).contiguous().float() for k, v in out.items()}


def make_sequence(H: int, W: int, seed: int = 0, object_motion: float = 0.0, device="cpu",
                  **kw) -> SyntheticSequence:
    return SyntheticSequence(SceneSpec(H=H, W=W, seed=seed, object_motion=object_motion, **kw),
                             device=device)


def random_band(shape, generator: torch.Generator, device="cpu") -> torch.Tensor:
    """Band input for standalone spatial-filter tests: 1/(x^2 + 1e-4) with
    x ~ N(0, 1), the network head's mapping (scripts/main.py:112), clipped to
    1e4."""
    x = torch.randn((*shape[:3], 5), generator=generator, device=device)
    return (1.0 / (x * x + 1e-4)).clamp(max=1e4)
