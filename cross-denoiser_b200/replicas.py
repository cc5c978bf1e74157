"""Multi-GPU plumbing of the denoiser: replicas, no data-path collective.

Every camera stream is independent (its own history, network weights and
Adam state), so N GPUs run N independent sets of streams, one process per
GPU.  The only communication is for measurement: the job's time is the
maximum over ranks.  `shard` assigns streams to ranks so that every rank
gets about the same number of pixels per frame round.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import torch
import torch.distributed as dist


def shard(resolutions: Sequence[Tuple[int, int]], world: int) -> List[List[int]]:
    """Stream ids per rank: largest streams first, each to the rank with the
    fewest pixels so far (ties to the lower rank).  Deterministic."""
    order = sorted(range(len(resolutions)), key=lambda s: (-resolutions[s][0] * resolutions[s][1], s))
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for s in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(s)
        load[r] += resolutions[s][0] * resolutions[s][1]
    return [sorted(x) for x in out]


def max_over_ranks(x: float) -> float:
    """Maximum of x over the process group (x itself without one).  Every
    rank must call it at the same point."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
