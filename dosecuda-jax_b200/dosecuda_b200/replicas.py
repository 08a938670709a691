"""Independent plans on several GPUs: one process per GPU, no data-path
collective (the pencil-beam path shards by plan and by beam; a plan fits
one GPU).  This module holds the host bookkeeping: process-group set-up
from the launcher's environment, a balanced split of plans over ranks,
and the max / sum reductions used to report the slowest rank's time and
the whole job's work.  The reference is single-GPU (gpu_id per call,
DoseCUDA/dose_kernels/IMPTClasses.cu:276,303).
"""
from __future__ import annotations

import datetime
import os
from typing import Tuple

import torch


def env_ranks() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the torch.distributed launcher."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> Tuple[int, int, int]:
    """Join the process group when the job has more than one rank.  With
    NCCL each rank binds its local GPU first.  A short timeout makes ranks
    that wait for a missing peer fail instead of hanging."""
    import torch.distributed as dist
    world, rank, local = env_ranks()
    if world > 1 and not dist.is_initialized():
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, **kw)
    return world, rank, local


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous share of n_items for `rank`; sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def _reduce(x: float, world: int, op, device) -> float:
    if world == 1:
        return float(x)
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, world: int, device=None) -> float:
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.MAX if world > 1 else None, device)


def sum_over_ranks(x: float, world: int, device=None) -> float:
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.SUM if world > 1 else None, device)


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def finish(world: int) -> None:
    """Leave the process group (every rank takes the same final barrier)."""
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.barrier()
            dist.destroy_process_group()
