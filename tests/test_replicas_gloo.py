"""Host logic of the multi-GPU bench (replicas: one process per GPU, each scoring its own share
of the guides on its own index copy; timings reduced as the max over ranks), run as two gloo
ranks on the CPU. No GPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert bench.dist_env() == (world, rank, rank)
        allq = np.arange(world * 1000, dtype=np.uint64) * 7919
        mine = bench.rank_share(allq, rank, 1000)
        ms = 10.0 + 5.0 * rank  # this rank's timed region
        worst = bench.max_over_ranks(ms)
        dist.barrier()
        out[rank] = (mine[0], mine[-1], len(mine), worst,
                     bench.whole_job_rate(world, 1000, 4, worst / 1e3))
    finally:
        dist.destroy_process_group()


def test_two_replicas_share_guides_and_take_the_slowest_rank():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    allq = np.arange(world * 1000, dtype=np.uint64) * 7919
    (a0, a1, n0, w0, r0), (b0, b1, n1, w1, r1) = out[0], out[1]
    assert (a0, a1, n0) == (allq[0], allq[999], 1000)
    assert (b0, b1, n1) == (allq[1000], allq[1999], 1000)  # disjoint shares covering the set
    assert w0 == w1 == 15.0                                 # every rank sees the slowest rank's time
    assert r0 == r1 == world * 1000 * 4 / 0.015             # whole-job guides/s
