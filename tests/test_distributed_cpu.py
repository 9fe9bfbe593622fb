"""Source-sharded Brandes across ranks (world size 2, gloo, CPU): the
all-reduced sum of per-shard betweenness equals the single-process result.
The per-shard compute here is the CPU oracle standing in for a GPU per rank;
the sharding and the reduction are the library's (zog_b200.distributed)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, V, frm, to, out):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle as O
        from zog_b200.distributed import betweenness_sharded

        ag = O.ArrayGraph(V, frm, to)

        def partial(src):
            bc, _ = ag.betweenness_sources(src)
            return torch.from_numpy(bc.copy())

        bc = betweenness_sharded(partial, np.arange(V, dtype=np.uint32), rank, world)
        out[rank] = bc.numpy().tobytes()
    finally:
        dist.destroy_process_group()


def test_sharded_betweenness_equals_full(oracle):
    V, f, t = oracle.rmat(9, 8, 909, directed=False)
    full, _ = oracle.ArrayGraph(V, f, t).betweenness_unweighted()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, V, f, t, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        bc = np.frombuffer(out[r], dtype=np.float64)
        assert np.abs(bc - full).sum() <= 1e-12 * np.abs(full).sum()


def test_shard_sources_partition():
    from zog_b200.distributed import shard_sources

    src = np.arange(103, dtype=np.uint32)
    parts = [shard_sources(src, r, 4) for r in range(4)]
    assert sorted(np.concatenate(parts).tolist()) == src.tolist()
    with pytest.raises(ValueError):
        shard_sources(src, 4, 4)
