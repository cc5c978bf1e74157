"""Helpers for the GPU tests: host <-> device conversion and seeded frames."""
import numpy as np
import pytest
import torch

from oracle import reference as ref


def T(a, dev="cuda:0"):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def N(t):
    return t.detach().cpu().numpy()


def frames(cd, H, W, seed=0, motion=2.0, t=5):
    seq = cd.synth.make_sequence(H, W, seed=seed, object_motion=motion)
    f0 = {k: v.numpy() for k, v in seq.frame(t - 1).items()}
    f1 = {k: v.numpy() for k, v in seq.frame(t).items()}
    return f0, f1


def batch(*frames_list):
    """Stack B single-frame dicts into [B,H,W,C] arrays."""
    return {k: np.concatenate([f[k] for f in frames_list], 0) for k in frames_list[0]}


needs_reference = pytest.mark.skipif(not ref.available(),
                                     reason="reference kernels (oracle/_ref) not built")
