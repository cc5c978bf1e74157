"""Reproject on the GPU: bit-exact success masks and outputs within 1e-4 of
the oracle, of the golden reference outputs and of the live reference
kernel; the generic tensor-list path; edge cases and argument errors."""
import numpy as np
import pytest
import torch

from gpu_util import N, T, batch, frames, needs_reference
from helpers import assert_close, assert_equal, golden, golden_names
from oracle import oracle as orc
from oracle import reference as ref

pytestmark = pytest.mark.gpu
KEYS = ("mvec", "linear_z", "prev_linear_z", "normal", "prev_normal", "pn_fwidth", "opacity", "prev_opacity")


def run(cd, d, lists):
    s, outs = cd.ops.Reproject(T(d["mvec"]), [T(x) for x in lists], T(d["linear_z"]), T(d["prev_linear_z"]),
                               T(d["normal"]), T(d["prev_normal"]), T(d["pn_fwidth"]), T(d["opacity"]),
                               T(d["prev_opacity"]))
    torch.cuda.synchronize()
    assert s.dtype == torch.bool
    return N(s), [N(o) for o in outs]


def seq_inputs(cd, H, W, seed, B=1):
    fs = [frames(cd, H, W, seed=seed + b, motion=2.0) for b in range(B)]
    f0 = batch(*[f[0] for f in fs])
    f1 = batch(*[f[1] for f in fs])
    d = dict(mvec=f1["mvec"], linear_z=f1["linearZ"], prev_linear_z=f0["linearZ"], normal=f1["normal"],
             prev_normal=f0["normal"], pn_fwidth=f1["pnFwidth"], opacity=f1["opacity"].copy(),
             prev_opacity=f0["opacity"].copy())
    d["opacity"][:, 3:7, 5:40] = 0.0
    d["prev_opacity"][:, 30:40, 60:70] = 0.0
    lists = [np.log1p(f0["color"]), np.log1p(f0["color2"]), f0["albedo"]]
    return d, lists


@pytest.mark.parametrize("name", golden_names("reproject_"))
def test_golden(cd, cuda, name):
    g = golden(name)
    d = {k: g["in_" + k] for k in KEYS}
    lists = [g[k] for k in sorted(k for k in g if k.startswith("in_list"))]
    s, outs = run(cd, d, lists)
    assert_equal(s, g["ref_success"], f"{name} success")
    for i, o in enumerate(outs):
        assert_close(o, g[f"ref_out{i}"], f"{name} out{i}")


@pytest.mark.parametrize("H,W,B", [(256, 256, 2), (67, 93, 1)])
def test_sequence_vs_oracle(cd, cuda, H, W, B):
    d, lists = seq_inputs(cd, H, W, seed=20, B=B)
    s, outs = run(cd, d, lists)
    rs, routs = orc.reproject(d["mvec"], lists, *[d[k] for k in KEYS[1:]])
    assert 0.5 < rs.mean() < 1.0
    assert_equal(s, rs, "success")
    for i in range(3):
        assert_close(outs[i], routs[i], f"out{i}")


def test_generic_list(cd, cuda):
    d, lists = seq_inputs(cd, 64, 80, seed=4)
    rng = np.random.default_rng(0)
    lists = [lists[0], rng.uniform(size=(1, 64, 80, 1)).astype(np.float32),
             rng.uniform(size=(1, 64, 80, 5)).astype(np.float32)]
    s, outs = run(cd, d, lists)
    rs, routs = orc.reproject(d["mvec"], lists, *[d[k] for k in KEYS[1:]])
    assert_equal(s, rs, "success")
    for i in range(3):
        assert outs[i].shape == lists[i].shape
        assert_close(outs[i], routs[i], f"out{i}")


def test_production_size_mask(cd, cuda):
    d, lists = seq_inputs(cd, 1080, 1920, seed=33)
    s, outs = run(cd, d, lists)
    rs, routs = orc.reproject(d["mvec"], lists, *[d[k] for k in KEYS[1:]])
    assert_equal(s, rs, "success 1080p")
    assert_close(outs[0], routs[0], "out0 1080p")


@needs_reference
def test_vs_reference_kernel(cd, cuda):
    d, lists = seq_inputs(cd, 256, 320, seed=7, B=2)
    s, outs = run(cd, d, lists)
    rs, routs = ref.reproject(T(d["mvec"]), [T(x) for x in lists], *[T(d[k]) for k in KEYS[1:]])
    torch.cuda.synchronize()
    assert_equal(s, N(rs), "success vs reference")
    for i in range(3):
        assert_close(outs[i], N(routs[i]), f"out{i} vs reference")


def test_edge_cases(cd, cuda):
    d, lists = seq_inputs(cd, 32, 48, seed=2)
    # all-zero opacity: everything rejected, outputs zero
    d0 = dict(d, opacity=np.zeros_like(d["opacity"]))
    s, outs = run(cd, d0, lists)
    assert not s.any() and all(np.all(o == 0) for o in outs)
    # motion far off screen: everything rejected
    d1 = dict(d, mvec=np.full_like(d["mvec"], 3.0))
    s, _ = run(cd, d1, lists)
    assert not s.any()
    # one-pixel and one-row images
    for H, W in ((1, 1), (1, 17), (9, 1)):
        dd = {k: v[:, :H, :W].copy() for k, v in d.items()}
        ll = [x[:, :H, :W].copy() for x in lists]
        s, outs = run(cd, dd, ll)
        rs, routs = orc.reproject(dd["mvec"], ll, *[dd[k] for k in KEYS[1:]])
        assert_equal(s, rs, f"success {H}x{W}")


def test_argument_errors(cd, cuda):
    d, lists = seq_inputs(cd, 16, 16, seed=1)
    a = [T(d[k]) for k in KEYS]
    with pytest.raises(ValueError):
        cd.ops.Reproject(a[0], [], *a[1:])
    with pytest.raises(ValueError):
        cd.ops.Reproject(a[0], [T(lists[0])] * 9, *a[1:])
    with pytest.raises(ValueError):
        cd.ops.Reproject(a[0], [T(lists[0][:, :8])], *a[1:])
    with pytest.raises(ValueError):
        cd.ops.Reproject(a[0].double(), [T(lists[0])], *a[1:])


def test_depth_ratio_boundary(cd, cuda):
    """Depth differences within a few ulps of the reference's threshold
    |Zp - Z| / (fwidthZ + 1e-2f) > 10 (ops/reproject.cu.cc:42), which the
    kernel decides without dividing: the previous depth is 0 everywhere and
    every pixel's |Z| sits k ulps from 10 (fwidthZ + 1e-2), k in -4..4, so all
    its taps (and its 3x3 fallback) take the same decision; the mask equals
    the oracle's, which divides."""
    rng = np.random.default_rng(11)
    B, H, W = 1, 64, 96
    fw = rng.uniform(0.0, 2.0, (B, H, W)).astype(np.float32)
    den = (fw + np.float32(1e-2)).astype(np.float32)
    k = rng.integers(-4, 5, (B, H, W))
    z = np.float32(10.0) * den
    z = np.nextafter(z, np.where(k > 0, np.float32(np.inf), np.float32(-np.inf)), dtype=np.float32)
    for _ in range(3):   # up to 4 ulps either way
        more = np.abs(k) > 1
        z = np.where(more, np.nextafter(z, np.where(k > 0, np.float32(np.inf), np.float32(-np.inf)),
                                        dtype=np.float32), z)
        k = np.where(more, k - np.sign(k), k)
    z = np.where(k == 0, np.float32(10.0) * den, z).astype(np.float32)
    lin = np.stack([z, fw, np.zeros_like(z)], -1).astype(np.float32)
    n = np.broadcast_to(np.array([0.0, 0.6, 0.8], np.float32), (B, H, W, 3)).copy()
    d = dict(mvec=np.zeros((B, H, W, 3), np.float32), linear_z=lin, prev_linear_z=np.zeros_like(lin),
             normal=n, prev_normal=n.copy(), pn_fwidth=np.zeros((B, H, W, 3), np.float32),
             opacity=np.ones((B, H, W, 1), np.float32), prev_opacity=np.ones((B, H, W, 1), np.float32))
    lists = [rng.uniform(0, 1, (B, H, W, 3)).astype(np.float32)]
    s, _ = run(cd, d, lists)
    rs, _ = orc.reproject(d["mvec"], lists, *[d[kk] for kk in KEYS[1:]])
    inner = rs[:, 1:-1, 1:-1]
    assert 0.2 < inner.mean() < 0.8, "the inputs straddle the threshold"
    assert_equal(s, rs, "success at the depth-ratio boundary")
