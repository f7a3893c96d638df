"""The N > 1 host path of bench.py on CPU: two gloo ranks run disjoint leases (replicas, no data
exchange) and time the job as the maximum over ranks, as they do over NCCL on GPUs."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, steps: int, queue) -> None:
    import datetime
    import sys
    import torch.distributed as dist
    from conftest import ROOT
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group('gloo', init_method=f'tcp://127.0.0.1:{port}', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = [bench.lease_bounds(k * world + rank) for k in range(steps)]   # bench's step assignment
        every = [None] * world
        dist.all_gather_object(every, mine)
        bench.barrier(dist)
        worst = bench.max_over_ranks(dist, 1.0 + rank, 0)
        queue.put((rank, every, worst))
    finally:
        dist.destroy_process_group()


def test_two_ranks_run_disjoint_leases_and_report_the_slowest():
    import torch.multiprocessing as mp
    world, steps = 2, 3
    port = _free_port()
    ctx = mp.get_context('spawn')
    queue = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, steps, queue)) for r in range(world)]
    for p in procs:
        p.start()
    got = [queue.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import bench
    from psuedocubes_b200.optimized import LEASE_WIDTH
    for rank, every, worst in got:
        assert worst == float(world)                         # the max over ranks, seen by every rank
        leases = [lease for per_rank in every for lease in per_rank]
        assert len(set(leases)) == world * steps             # no lease runs twice
        assert all(end - first == LEASE_WIDTH for first, end in leases)
        firsts = sorted(first for first, _ in leases)
        assert all(b - a >= LEASE_WIDTH for a, b in zip(firsts, firsts[1:]))   # disjoint v ranges
        assert every[rank] == [bench.lease_bounds(k * world + rank) for k in range(steps)]
