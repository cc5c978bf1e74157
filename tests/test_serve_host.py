"""Scheduling logic of the serving loop (cross_denoiser_b200.serve) on the
CPU, with stand-in sessions: Poisson arrivals, in-order frames per stream,
one frame in flight per stream, concurrency across streams, admission by an
HBM budget with release on completion."""
import numpy as np

from cross_denoiser_b200 import serve


class FakeEvent:
    def __init__(self, polls):
        self.left = polls

    def query(self):
        self.left -= 1
        return self.left <= 0


class FakeSession:
    log = []

    def __init__(self, sid, H, W, src):
        self.sid, self.inflight, self.next_frame = sid, None, 0
        FakeSession.log.append(("admit", sid))

    def launch(self, frame, host=None):
        assert frame == self.next_frame, "frames of a stream run in order"
        FakeSession.log.append(("launch", self.sid, frame))
        self.next_frame = frame + 1
        return FakeEvent(3)

    def release(self):
        FakeSession.log.append(("release", self.sid))


def test_poisson_schedule():
    rates = [30.0, 120.0]
    sch = serve.poisson_schedule(rates, 2000, seed=1)
    assert [q.arrival for q in sch] == sorted(q.arrival for q in sch)
    for sid, r in enumerate(rates):
        t = np.array([q.arrival for q in sch if q.stream_id == sid])
        assert [q.frame for q in sch if q.stream_id == sid] == list(range(2000))
        assert abs(np.mean(np.diff(t)) * r - 1.0) < 0.08


def run_fake(budget, nstreams=4, frames=3, res=None):
    FakeSession.log = []
    res = res or [(8, 8)] * nstreams
    srv = serve.Server(res, lambda sid, t: None, "cpu", hbm_budget=budget, session_factory=FakeSession,
                       memory_probe=lambda: 0)
    srv.measured = {r: 100 for r in set(res)}
    sch = serve.poisson_schedule([1000.0] * len(res), frames, seed=2)
    out = srv.run(sch, frames, realtime=False)
    return srv, out


def test_all_streams_concurrent_when_budget_allows():
    srv, out = run_fake(budget=10_000)
    assert len(out) == 12 and srv.max_admitted == 4 and srv.admission_waits == 0
    # every stream launched its first frame before any stream launched a third
    launches = [e for e in FakeSession.log if e[0] == "launch"]
    first3 = min(i for i, e in enumerate(launches) if e[2] == 2)
    assert {e[1] for e in launches[:first3] if e[2] == 0} == {0, 1, 2, 3}
    for sid in range(4):
        assert [r.frame for r in out if r.stream_id == sid] == [0, 1, 2]


def test_admission_waits_for_memory():
    srv, out = run_fake(budget=250)          # two streams of 100 bytes fit at a time
    assert len(out) == 12 and srv.max_admitted == 2 and srv.admission_waits > 0
    log = FakeSession.log
    # the third admission happens only after a release
    i3 = [i for i, e in enumerate(log) if e[0] == "admit"][2]
    assert any(e[0] == "release" for e in log[:i3])


def test_stream_larger_than_budget_is_refused():
    import pytest
    with pytest.raises(MemoryError):
        run_fake(budget=50)


def test_summarize():
    res = [(4, 4), (8, 8)]
    rs = [serve.Result(0, 0, 0.0, 0.0, 0.010), serve.Result(1, 0, 0.0, 0.0, 0.020),
          serve.Result(0, 1, 0.015, 0.015, 0.030)]
    s = serve.summarize(rs, res)
    assert s["frames"] == 3 and abs(s["seconds"] - 0.030) < 1e-9
    assert s["by_resolution"]["4x4"]["frames"] == 2 and s["by_resolution"]["8x8"]["frames"] == 1


def test_session_failure_stops_the_loop():
    """A session whose check() raises (its network reported a time-out) ends
    the run with that error once its frame completes."""
    class Boom(RuntimeError):
        pass

    class Failing(FakeSession):
        def check(self):
            if self.next_frame >= 2:
                raise Boom(f"stream {self.sid}")

    srv = serve.Server([(8, 8)] * 2, lambda sid, t: None, "cpu", hbm_budget=1 << 30, session_factory=Failing,
                       memory_probe=lambda: 0)
    import pytest
    with pytest.raises(Boom):
        srv.run(serve.poisson_schedule([50.0, 50.0], 4, seed=2), 4, realtime=False)


def test_admit_all_and_warm_then_run():
    """Streams admitted and warmed before the timed run continue from the
    warm frames: run() serves only the later frames, in order, and retires
    every stream."""
    FakeSession.log = []
    res = [(8, 8)] * 3
    srv = serve.Server(res, lambda sid, t: None, "cpu", hbm_budget=1 << 30, session_factory=FakeSession,
                       memory_probe=lambda: 0)
    assert srv.admit_all() == 3
    srv.warm(2)
    sched = [q for q in serve.poisson_schedule([40.0] * 3, 5, seed=4) if q.frame >= 2]
    results = srv.run(sched, 5, realtime=False)
    assert sorted((r.stream_id, r.frame) for r in results) == [(s, t) for s in range(3) for t in range(2, 5)]
    assert all(("admit", s) in FakeSession.log for s in range(3))
    assert [e for e in FakeSession.log if e[0] == "admit"] == [("admit", 0), ("admit", 1), ("admit", 2)]
    assert set(srv.retired) == {0, 1, 2}
