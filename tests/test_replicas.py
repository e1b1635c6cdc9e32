"""Multi-replica host logic on CPU ranks (gloo, world size 2): frame split,
max-over-ranks timing and the gradient all-reduce of the adjoint."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from falcor_b200.replicas import allreduce_gradients, frame_seeds, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        seeds = frame_seeds(rank, world, 16)
        t = max_over_ranks(10.0 + rank)
        g = torch.full((5,), float(rank + 1))
        p = torch.arange(3, dtype=torch.float32) * (rank + 1)
        allreduce_gradients(g, None, p)
        out.put((rank, seeds, t, g.tolist(), p.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_cpu_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seeds = [r[1] for r in res]
    assert sorted(seeds[0] + seeds[1]) == list(range(16)) and not set(seeds[0]) & set(seeds[1])
    assert all(r[2] == 11.0 for r in res)
    assert all(r[3] == [3.0] * 5 for r in res)
    assert all(r[4] == [0.0, 3.0, 6.0] for r in res)


def test_single_process_is_identity():
    from falcor_b200.replicas import allreduce_gradients, frame_seeds, max_over_ranks
    assert frame_seeds(0, 1, 4, base=10) == [10, 11, 12, 13]
    assert max_over_ranks(2.5) == 2.5
    g = torch.ones(3)
    allreduce_gradients(g)
    assert g.tolist() == [1.0, 1.0, 1.0]
