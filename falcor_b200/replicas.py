"""Multi-GPU replicas (one process per GPU, torch.distributed).

Paths are independent, so the forward path runs as independent replicas with no
data-path collective (weak scaling); the adjoint has one exchange: the gradient
buffers of the replicas are summed (ncclAllReduce over NVLink with the "nccl"
backend), as a multi-GPU inverse-rendering loop needs.  Timing across ranks is
the maximum over ranks.
"""
from __future__ import annotations


def frame_seeds(rank: int, world: int, frames: int, base: int = 0) -> list[int]:
    """Frame seeds of one rank when `frames` frames are split across `world`
    replicas: rank r renders frames r, r + world, ... (disjoint, covering)."""
    return [base + f for f in range(rank, frames, world)]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (e.g. a timed duration) over all ranks."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_world() -> tuple[int, int]:
    """(rank, world size) of the default process group, (0, 1) without one."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(items, rank: int | None = None, world: int | None = None) -> list:
    """This rank's share of a list of independent work items (requests, views,
    frames): items rank, rank + world, ... as (index, item) pairs, so that the
    ranks' shares are disjoint and cover the list."""
    if rank is None or world is None:
        rank, world = rank_world()
    return [(i, items[i]) for i in range(rank, len(items), world)]


def sharded_sum(items, fn, like=None):
    """Sum over all ranks of fn(index, item) for the items of a list: each rank
    calls fn on its shard (``shard``), sums the returned tuples of tensors
    element by element, and the sums are all-reduced (the only data-path
    collective of a multi-GPU adjoint: gradient buffers summed over NVLink).
    ``like`` gives zero tensors for a rank whose shard is empty.  Returns the
    tuple of summed tensors, identical on every rank."""
    acc = None
    for i, item in shard(items):
        out = tuple(fn(i, item))
        acc = out if acc is None else tuple(a + b for a, b in zip(acc, out))
    if acc is None:
        if like is None:
            raise ValueError("sharded_sum: empty shard and no zero template")
        acc = tuple(t.clone() for t in like)
    acc = tuple(a.contiguous() for a in acc)
    allreduce_gradients(*acc)
    return acc


def allreduce_gradients(*grads) -> None:
    """Sums gradient tensors over all ranks in place (one collective per tensor)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return
    for g in grads:
        if g is not None:
            dist.all_reduce(g, op=dist.ReduceOp.SUM)
