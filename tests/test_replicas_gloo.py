"""Multi-process (world size 2, gloo, CPU) checks of the sharding / reduction plumbing."""
import os
import socket

import numpy as np
import pytest

from distorteddustydiscanalysistoolkits_b200 import replicas


def test_query_shard_partition():
    for npts in (0, 1, 7, 4194304):
        for world in (1, 2, 3, 8):
            cover = []
            for r in range(world):
                lo, hi = replicas.query_shard(npts, r, world)
                cover.extend(range(lo, hi)) if npts < 100 else cover.append((lo, hi))
            if npts < 100:
                assert cover == list(range(npts))
            else:
                assert cover[0][0] == 0 and cover[-1][1] == npts
                assert all(cover[i][1] == cover[i + 1][0] for i in range(world - 1))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mx = replicas.max_over_ranks([float(rank), 10.0 - rank])
        npts = 11
        lo, hi = replicas.query_shard(npts, rank, world)
        full = replicas.gather_shards(np.arange(lo, hi, dtype=np.float64) * 2.0, npts, rank, world)
        q.put((rank, mx, full.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, full in res:
        assert mx == [1.0, 10.0]
        assert full == [2.0 * i for i in range(11)]
