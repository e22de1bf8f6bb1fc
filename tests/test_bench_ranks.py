"""The multi-rank plumbing of bench.py (replicas, one process per GPU) on CPU: two gloo
ranks take the same barrier and max-over-ranks steps as NCCL ranks do on GPUs, and the
reference arm runs on rank 0 only."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime
    import sys
    from pathlib import Path
    import torch.distributed as dist
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier_sync(world)
        # each rank's time differs; every rank must get the slowest one
        out[rank] = bench.max_over_ranks(10.0 + rank, world)

        class Args:
            workload = 'dipole_core'
        # the reference arm: ranks other than 0 return without work
        if rank != 0:
            out[world + rank] = bench.run_reference(Args()) is None
        else:
            out[world + rank] = True
        bench.barrier_sync(world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world = 2
    port = _free_port()
    with mp.get_context('spawn').Manager() as m:  # no fork of this multi-threaded process
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        assert [out[r] for r in range(world)] == [11.0, 11.0]
        assert all(out[world + r] for r in range(world))
