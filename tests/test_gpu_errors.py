"""Error paths of the tensor-core kernels on the GPU, without a faulty kernel.

* The bounded mbarrier wait that the U-Net kernels use runs out on a barrier
  that nothing arrives at (no copy or MMA in flight), sets the error flag
  and returns; the context stays usable.  With an arrival the same wait
  completes and leaves the flag alone.
* A nonzero U-Net workspace flag (written by the test, as a timed-out
  kernel would write it) reaches the host through the asynchronous
  read-back: the network's next forward, the frame step and the serving
  loop raise UNetTimeoutError instead of going on with invalid outputs.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _probe(cd, arrive, max_iter):
    L = cd._lib.lib()
    flag = torch.zeros((1,), dtype=torch.int32, device="cuda:0")
    rc = L.cd_mbar_timeout_probe(ctypes.c_void_p(flag.data_ptr()), arrive, max_iter,
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.cd_get_last_error()
    torch.cuda.synchronize()
    return int(flag.item())


def test_bounded_wait_runs_out_and_sets_the_flag(cd, cuda):
    assert _probe(cd, arrive=0, max_iter=256) == 1
    assert _probe(cd, arrive=1, max_iter=256) == 0
    assert _probe(cd, arrive=0, max_iter=1) == 1
    # the context is still usable after the time-out
    x = torch.arange(1024, device=cuda, dtype=torch.float32)
    assert float(x.sum()) == 1023 * 1024 / 2
    L = cd._lib.lib()
    assert L.cd_mbar_timeout_probe(None, 0, 8, None) == cd._lib.CD_EINVAL
    assert L.cd_mbar_timeout_probe(ctypes.c_void_p(16), 0, 1 << 20, None) == cd._lib.CD_EINVAL


def _frames(cd, H, W, n, seed, cuda):
    seq = cd.synth.make_sequence(H, W, seed=seed, object_motion=2.0)
    return [{k: v.to(cuda) for k, v in seq.frame(t).items() if k in cd.synth.FRAME_INPUTS} for t in range(n)]


def _set_flag(net, value):
    net.ws[:4].view(torch.int32).fill_(value)


def test_unet_flag_stops_the_frame_step(cd, cuda):
    H, W = 64, 96
    fr = _frames(cd, H, W, 3, 31, cuda)
    net = cd.unet.UNet(cuda, seed=4)
    st = cd.step.FrameStep(cd.step.StepConfig(regression_width=9, filter_width=7, fused=True),
                           predictor=net, on_gradients=net.on_gradients)
    st(fr[0])
    torch.cuda.synchronize()
    assert net.error_flag() == 0
    net.raise_if_failed()
    # as a kernel that gave up on an MMA batch would leave it
    _set_flag(net, 2)
    net.enqueue_error_readback()
    torch.cuda.synchronize()
    assert net.error_flag() == 2
    with pytest.raises(cd.unet.UNetTimeoutError, match="flag 2"):
        st(fr[1])


def test_unet_flag_stops_the_serving_loop(cd, cuda):
    res = [(64, 96), (48, 64)]
    src = cd.serve.device_frame_source(res, [3, 4], cuda, pool=2)

    class Failing(cd.serve.Session):
        def _body(self):
            super()._body()
            if self.sid == 1:
                _set_flag(self.net, 1)

    cfg = cd.step.StepConfig(regression_width=9, filter_width=7, fused=True)
    srv = cd.serve.Server(res, src, cuda, hbm_budget=8 << 30, cfg=cfg,
                          session_factory=lambda sid, H, W, s: Failing(sid, H, W, s, cuda, cfg, seed=sid))
    sch = cd.serve.poisson_schedule([100.0, 100.0], 3, seed=1)
    with pytest.raises(cd.unet.UNetTimeoutError, match="flag 1"):
        srv.run(sch, 3, realtime=False)
    torch.cuda.synchronize()
