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


def _inverse_worker(rank, world, port, out):
    """One rank of a sharded inverse-rendering step on CPU tensors: the views
    are split across the ranks, each rank's per-view 'gradients' (a
    deterministic function of the view index standing in for forward + adjoint)
    are summed and all-reduced, and every rank takes the same Adam step."""
    import torch.distributed as dist
    from falcor_b200.replicas import shard, sharded_sum
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        views = [f"view{v}" for v in range(5)]
        seen = []

        def view_grad(v, _):
            seen.append(v)
            g = torch.Generator().manual_seed(100 + v)
            return torch.tensor([float(v)]), torch.randn(7, 3, generator=g), torch.randn(4, generator=g)

        zeros = (torch.zeros(1), torch.zeros(7, 3), torch.zeros(4))
        loss, gp, gc = sharded_sum(views, view_grad, like=zeros)
        # A one-view list leaves rank 1 with an empty shard.
        (one,) = sharded_sum(views[:1], lambda v, _: (torch.ones(2) * (v + 3),), like=(torch.zeros(2),))
        x = torch.zeros(7, 3, requires_grad=True)
        opt = torch.optim.Adam([x], lr=1e-2)
        x.grad = gp.clone()
        opt.step()
        out.put((rank, seen, [i for i, _ in shard(views)], float(loss), gp.tolist(), gc.tolist(), one.tolist(),
                 x.detach().tolist()))
    finally:
        dist.destroy_process_group()


def test_two_cpu_ranks_sharded_inverse_step():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_inverse_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, seen0, sh0, loss0, gp0, gc0, one0, x0), (_, seen1, sh1, loss1, gp1, gc1, one1, x1) = res
    assert seen0 == sh0 == [0, 2, 4] and seen1 == sh1 == [1, 3]
    assert loss0 == loss1 == 10.0
    gens = [torch.Generator().manual_seed(100 + v) for v in range(5)]
    ref = [(torch.randn(7, 3, generator=g), torch.randn(4, generator=g)) for g in gens]
    gp_ref = sum(r[0] for r in ref)
    gc_ref = sum(r[1] for r in ref)
    assert gp0 == gp1 and gc0 == gc1 and x0 == x1
    assert torch.allclose(torch.tensor(gp0), gp_ref, atol=1e-5) and torch.allclose(torch.tensor(gc0), gc_ref, atol=1e-5)
    assert one0 == one1 == [3.0, 3.0]
