"""Serving on the GPU: streams of different resolutions run concurrently
(each on its own CUDA stream, CUDA-graph replay after the first frame) and
every frame's denoised output is the same as when the stream runs alone, and
the same as the eager per-frame step.  Tolerance: bit-identical (every
kernel is deterministic and streams share no state)."""
import numpy as np
import pytest
import torch

from gpu_util import N

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
RES = [(64, 96), (48, 64), (64, 96), (32, 128)]
FRAMES = 5


def server(cd, res, graphs=True, budget=8 << 30):
    seeds = [11 + 7 * i for i in range(len(res))]
    src = cd.serve.device_frame_source(res, seeds, DEV, pool=3)
    for sid in range(len(res)):
        src(sid, 0)
    cfg = cd.step.StepConfig(regression_width=9, filter_width=7, fused=True)
    return cd.serve.Server(res, src, DEV, hbm_budget=budget, cfg=cfg, graphs=graphs, keep_outputs=True, seed=5)


def outputs(srv, sid):
    return [N(t) for t in srv.retired[sid].outputs]


def test_mix_equals_alone_and_eager(cd, cuda):
    mix = server(cd, RES)
    sch = cd.serve.poisson_schedule([200.0] * len(RES), FRAMES, seed=3)
    res = mix.run(sch, FRAMES, realtime=False)
    assert len(res) == len(RES) * FRAMES
    assert mix.max_admitted == len(RES)
    for sid in range(len(RES)):
        got = outputs(mix, sid)
        assert len(got) == FRAMES
        # alone: a server holding only this stream (same seeds -> same stream)
        alone = server(cd, RES)
        one = [q for q in sch if q.stream_id == sid]
        alone.run(one, FRAMES, realtime=False)
        for t, (a, b) in enumerate(zip(got, outputs(alone, sid))):
            np.testing.assert_array_equal(a, b, err_msg=f"stream {sid} frame {t}: mix vs alone")
    # eager (no graphs) equals graph replay
    eager = server(cd, RES, graphs=False)
    eager.run(sch, FRAMES, realtime=False)
    for sid in range(len(RES)):
        for t, (a, b) in enumerate(zip(outputs(mix, sid), outputs(eager, sid))):
            np.testing.assert_array_equal(a, b, err_msg=f"stream {sid} frame {t}: graph vs eager")


def test_admission_under_budget(cd, cuda):
    srv = server(cd, RES)
    srv.calibrate(frames=2)
    assert all(v > 0 for v in srv.measured.values()) and len(srv.measured) == len(set(RES))
    # admission on round figures: 1 GiB per stream, 2.5 GiB budget -> at most two resident
    srv.measured = {r: 1 << 30 for r in set(RES)}
    srv.budget = int(2.5 * (1 << 30))
    sch = cd.serve.poisson_schedule([200.0] * len(RES), 3, seed=4)
    res = srv.run(sch, 3, realtime=False)
    assert len(res) == len(RES) * 3
    assert srv.max_admitted <= 2 and srv.admission_waits > 0
