"""One process per GPU: plane sharding and the host-side rank plumbing.

Every plane (level x field x member) is an independent transform, so N GPUs
run N replicas of the engine on N sets of planes with no collective on the
data path (the reference's multi-card transports, ``cards.py``, exist for
16 GB cards and are not needed here).  What the ranks do share is host-side:
which planes each one owns, the timing reduction (the step time of a job is
the slowest rank's), and, for a caller that wants every plane on one GPU
afterwards, one all-gather.  The functions take an optional process group
and work with any ``torch.distributed`` backend (NCCL on the GPUs, gloo in
the CPU tests).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_planes(total: int, rank: int, world: int) -> tuple[int, int]:
    """``(first, count)`` of rank ``rank``'s contiguous share of ``total``
    planes: the first ``total % world`` ranks hold one plane more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if total < 0:
        raise ValueError("total must be >= 0")
    base, extra = divmod(int(total), int(world))
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def world() -> tuple[int, int]:
    """``(rank, world_size)``, ``(0, 1)`` without an initialised group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The maximum of ``value`` over the ranks (the job's step time is the
    slowest rank's); the value itself on a single process."""
    rank, size = world()
    if size == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def barrier(device=None, group=None) -> None:
    """A barrier over the ranks (a no-op on a single process)."""
    _, size = world()
    if size > 1:
        if device is not None and torch.device(device).type == "cuda":
            dist.barrier(group=group, device_ids=[torch.device(device).index])
        else:
            dist.barrier(group=group)


def gather_planes(local: torch.Tensor, counts: list[int], group=None) -> torch.Tensor:
    """Concatenate every rank's planes (leading axis) in rank order.

    ``counts`` holds each rank's plane count (``shard_planes``); ranks with
    fewer planes are padded for the collective and trimmed afterwards."""
    rank, size = world()
    if size == 1:
        return local
    if len(counts) != size or local.shape[0] != counts[rank]:
        raise ValueError("counts must list every rank's plane count, this rank's matching `local`")
    width = max(counts)
    pad = torch.zeros((width, *local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(size)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)
