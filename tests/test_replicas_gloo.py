"""Multi-process path on the CPU: two gloo ranks, as bench.py runs one rank
per GPU.  Replicas only: the ranks exchange nothing but the max-over-ranks
timing; streams are sharded by pixel load."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _replicas():
    import __graft_entry__ as ge
    ge.load_package()
    from cross_denoiser_b200 import replicas
    return replicas

SERVE_RES = [(720, 1280)] * 4 + [(1080, 1920)] * 8 + [(1440, 2560)] * 3 + [(2160, 3840)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    replicas = _replicas()
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = replicas.max_over_ranks(1.5 + rank)
        mine = replicas.shard(SERVE_RES, world)[rank]
        # every rank computes the same assignment
        got = [None] * world
        dist.all_gather_object(got, mine)
        q.put((rank, t, got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = []
    for _ in range(world):
        res.append(q.get(timeout=120))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    replicas = _replicas()
    for rank, t, got in res:
        assert t == 1.5 + world - 1                     # the max over ranks
        assert got == replicas.shard(SERVE_RES, world)  # identical on every rank


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_covers_every_stream_once_and_balances(world):
    parts = _replicas().shard(SERVE_RES, world)
    flat = sorted(s for p in parts for s in p)
    assert flat == list(range(len(SERVE_RES)))
    px = [sum(SERVE_RES[s][0] * SERVE_RES[s][1] for s in p) for p in parts]
    biggest = max(h * w for h, w in SERVE_RES)
    assert max(px) - min(px) <= biggest


def test_single_process_is_identity():
    assert _replicas().max_over_ranks(3.25) == 3.25
