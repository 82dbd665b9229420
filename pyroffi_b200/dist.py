"""Data-parallel sharding of the path over ranks (one process per GPU).

Configurations, seeds, IK problems and trajectories are independent, so a
multi-GPU run splits the batch into contiguous ranges, one per rank, with the
robot and the obstacle set replicated on every GPU.  No collective runs on
the data path: each rank launches the same kernels on its own range.  Results
come back by one all-gather (NCCL on GPUs, gloo on CPU) when a caller wants
them on every rank, and timings are reduced with a max over ranks.
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def world() -> tuple[int, int]:
    """(rank, world_size); (0, 1) without an initialised process group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard_range(n: int, rank: int, world_size: int) -> tuple[int, int]:
    """Contiguous [start, stop) of ``n`` items for ``rank``; the first
    ``n % world_size`` ranks take one extra item."""
    if world_size <= 0 or not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside world of size {world_size}")
    if n < 0:
        raise ValueError("negative item count")
    base, extra = divmod(n, world_size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard(t: torch.Tensor, rank: int | None = None, world_size: int | None = None) -> torch.Tensor:
    """This rank's contiguous slice of ``t`` along dim 0."""
    r, w = world()
    rank = r if rank is None else rank
    world_size = w if world_size is None else world_size
    a, b = shard_range(int(t.shape[0]), rank, world_size)
    return t[a:b]


def gather_shards(local: torch.Tensor, n_total: int) -> torch.Tensor:
    """Concatenate every rank's shard (ranks in order) into [n_total, ...] on every rank."""
    rank, w = world()
    if w == 1:
        return local
    sizes = [shard_range(n_total, r, w) for r in range(w)]
    cap = max(b - a for a, b in sizes)
    pad = torch.zeros((cap,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(w)]
    dist.all_gather(bufs, pad)
    return torch.cat([bufs[r][: b - a] for r, (a, b) in enumerate(sizes)], dim=0)


def max_over_ranks(seconds: float, device: torch.device | str = "cpu") -> float:
    """The slowest rank's time (every rank gets the same value)."""
    _, w = world()
    if w == 1:
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
