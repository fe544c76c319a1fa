"""Multi-process helpers for running the builder on several GPUs of one node.

Diagram construction shards without any data-path exchange: cells (and whole
point clouds) are independent, so every rank builds its own diagrams and the
only collective is the timing reduction (max over ranks). One process per GPU,
launched by torch.distributed.run; rendezvous from the environment
(RANK / WORLD_SIZE / LOCAL_RANK / MASTER_ADDR / MASTER_PORT).
"""

from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_world() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the launcher's environment (1 process if unset)."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init(backend: str, timeout_s: float = 120.0) -> tuple[int, int, int]:
    rank, world, local = env_world()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def shard_range(n_items: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block [begin, end) of n_items owned by `rank` (sizes differ by at most one)."""
    base, rem = divmod(n_items, world)
    begin = rank * base + min(rank, rem)
    return begin, begin + base + (1 if rank < rem else 0)


def reduce_max(value: float, device: torch.device | str = "cpu") -> float:
    """Max of a scalar over all ranks (identity without a process group)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, device: torch.device | str = "cpu") -> float:
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier() -> None:
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def finalize() -> None:
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
