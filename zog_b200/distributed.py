"""Multi-GPU plumbing for the two paths (one process per GPU, torch.distributed).

The reference has no distributed runtime; these are the two ways this library
spreads work over N GPUs of one node:

* Brandes shards the *sources*: every rank holds the whole graph, runs the
  sources r, r+N, r+2N, ... (`shard_sources`) and the partial score vectors
  are summed with one all-reduce (`betweenness_sharded`) -- the dependencies of
  different sources are independent and add up, so this is the real exchange
  step of the algorithm (centrality.zig:728-788 sums delta_s over s).
* PageRank runs as independent replicas: every power iteration needs the whole
  previous vector, so a single graph of the benchmark size stays on one GPU.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def shard_sources(sources, rank: int, world: int) -> np.ndarray:
    """Sources of one rank: a strided slice, so hubs and leaves mix evenly."""
    src = np.asarray(sources, dtype=np.uint32)
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    return src[rank::world]


def betweenness_sharded(partial: Callable[[np.ndarray], "object"], sources, rank: int, world: int, group=None):
    """Sum over ranks of `partial(my_sources)`.

    `partial` returns this rank's betweenness vector (a torch tensor, on the
    device for NCCL or on the CPU for gloo) over its source shard; the result
    is the all-reduced sum, identical on every rank.
    """
    import torch.distributed as dist

    mine = shard_sources(sources, rank, world)
    bc = partial(mine)
    if world > 1:
        dist.all_reduce(bc, op=dist.ReduceOp.SUM, group=group)
    return bc
