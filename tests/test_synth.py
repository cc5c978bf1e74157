"""The seeded synthetic frame generator (stand-in for the reference's EXR
dataset): layout, value ranges and determinism."""
import numpy as np
import torch

from cross_denoiser_b200 import synth


def test_layout_and_ranges():
    seq = synth.make_sequence(40, 56, seed=3, object_motion=2.0)
    f = seq.frame(2)
    for k, c in synth.BUFFERS.items():
        assert f[k].shape == (1, 40, 56, c) and f[k].dtype == torch.float32
    assert (f["color"] > 0).all() and (f["color2"] > 0).all()
    assert f["albedo"].min() >= 0.05 and f["albedo"].max() <= 0.95
    n = f["normal"].norm(dim=-1)
    assert torch.allclose(n, torch.ones_like(n), atol=1e-5)
    z = f["linearZ"][..., 0]
    assert z.min() >= 1 and z.max() <= 50
    assert (f["linearZ"][..., 2] == 0).all() and (f["mvec"][..., 2] == 0).all()
    assert (f["opacity"] == 1).all()
    motion_px = f["mvec"][..., 0] * 56
    assert motion_px.abs().max() < 3.5 + 2.0


def test_deterministic():
    a = synth.make_sequence(24, 32, seed=9).frame(5)
    b = synth.make_sequence(24, 32, seed=9).frame(5)
    c = synth.make_sequence(24, 32, seed=10).frame(5)
    for k in a:
        assert torch.equal(a[k], b[k])
    assert not torch.equal(a["color"], c["color"])


def test_fireflies_and_sparse_hdr():
    f = synth.make_sequence(128, 128, seed=1).frame(0)
    frac = (f["emissive"].amax(-1) > 0).float().mean().item()
    assert 0.01 < frac < 0.03


def test_band_mapping():
    g = torch.Generator().manual_seed(0)
    b = synth.random_band((1, 8, 8), g)
    assert b.shape == (1, 8, 8, 5) and b.min() > 0 and b.max() <= 1e4
