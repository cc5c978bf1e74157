"""The NPY scene layout of the reference's DataLoader (scripts/utils.py:
147-305) on the CPU: a synthetic sequence written as {type}_{frame:04d}.npy
reads back bit for bit; the loader's validation (missing type, different
frame sets, EXR-only directories), frame wrapping and skip_frames; NaN/Inf
sanitisation; the driver's output composition and relL2."""
import os

import numpy as np
import pytest
import torch


def _write(cd, tmp_path, n=3, H=16, W=24):
    seq = cd.synth.make_sequence(H, W, seed=5, object_motion=1.0)
    frames = [seq.frame(t) for t in range(n)]
    cd.frames.save_npy_sequence(str(tmp_path), frames, start=0)
    return frames


def test_round_trip(cd, tmp_path):
    frames = _write(cd, tmp_path)
    seq = cd.frames.NpySequence(str(tmp_path), types=cd.frames.STEP_TYPES, pin=False)
    assert len(seq) == 3 and seq.start_frame == 0
    for i, (t, f) in enumerate(seq):
        assert t == i
        for k in cd.frames.STEP_TYPES:
            assert f[k].dtype == torch.float32 and f[k].shape == frames[i][k].shape
            assert torch.equal(f[k], frames[i][k]), k
    # item indices wrap over the sequence, as the reference's loader does
    assert seq[4][0] == 1
    seq.skip_frames(1)
    assert len(seq) == 2 and seq[0][0] == 1
    got = [t for t, _ in seq.prefetch(depth=2)]
    assert got == [1, 2]


def test_validation(cd, tmp_path):
    _write(cd, tmp_path)
    with pytest.raises(ValueError, match="not given"):
        cd.frames.NpySequence(str(tmp_path), types=("color", "ref"), pin=False)
    os.remove(os.path.join(tmp_path, "albedo_0002.npy"))
    with pytest.raises(ValueError, match="different number"):
        cd.frames.NpySequence(str(tmp_path), pin=False)
    # frames at or beyond max_num_frames are ignored
    seq = cd.frames.NpySequence(str(tmp_path), max_num_frames=2, pin=False)
    assert len(seq) == 2
    exr = tmp_path / "exr"
    exr.mkdir()
    (exr / "color_0000.exr").write_bytes(b"")
    with pytest.raises(RuntimeError, match="EXR"):
        cd.frames.NpySequence(str(exr), types=("color",), pin=False)


def test_sanitised_and_metrics(cd, tmp_path):
    a = np.ones((1, 4, 4, 3), np.float32)
    a[0, 0, 0, 0], a[0, 1, 1, 1], a[0, 2, 2, 2] = np.nan, np.inf, -np.inf
    np.save(tmp_path / "color_0000.npy", a)
    f = cd.frames.NpySequence(str(tmp_path), types=("color",), pin=False).frame(0)["color"]
    assert torch.isfinite(f).all() and float(f[0, 0, 0, 0]) == 0.0 and float(f[0, 1, 1, 1]) == 0.0
    out = torch.full((1, 2, 2, 3), 0.5)
    comp = cd.frames.compose_output(out, torch.full_like(out, 0.25), torch.full_like(out, 0.25))
    assert torch.equal(comp, torch.ones_like(out))
    ref = torch.rand((1, 4, 4, 3))
    pred = ref + 0.1
    e = cd.frames.rel_l2(pred, ref)
    want = 0.01 / (ref.mean(-1, keepdim=True) ** 2 + 1e-2)
    torch.testing.assert_close(e, want.expand_as(e), rtol=1e-5, atol=1e-7)
