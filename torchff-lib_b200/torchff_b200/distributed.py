"""Host-side multi-rank helpers (one process per GPU, torch.distributed).

Independent units (frames of a trajectory, serving requests, replica boxes) are split
across ranks with no data-path collective; the one exchange on the path is the sum of
parameter gradients over the frames of a force-matching step. Every rank calls these in
the same order.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def frame_shard(nframes: int, rank: int, world: int) -> list[int]:
    """Frames of this rank: rank, rank + world, ... (the union over ranks is every frame once)."""
    return list(range(rank, nframes, world))


def allreduce_sum_(tensors: list[torch.Tensor]) -> None:
    """In-place sum over ranks of several tensors with one collective (flattened copy)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat)
    off = 0
    for t in tensors:
        n = t.numel()
        t.copy_(flat[off:off + n].view_as(t))
        off += n


def max_over_ranks(value: float, device) -> float:
    """Largest value over ranks (timings: the job ends with its slowest rank)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
