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


def allreduce_gradients(*grads) -> None:
    """Sums gradient tensors over all ranks in place (one collective per tensor)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return
    for g in grads:
        if g is not None:
            dist.all_reduce(g, op=dist.ReduceOp.SUM)
