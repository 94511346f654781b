"""Multi-GPU replicas: independent integrations per rank, no data-path collective.

The barotropic path does not shard (all six faces of a member live on one GPU
and nothing crosses GPUs), so several GPUs run independent integrations: one
member per rank for the drop-in benchmark, or a share of an ensemble / of a
request stream per rank.  This module holds the plumbing: process-group set
up from the torchrun environment (NCCL between GPUs, gloo on CPU for tests),
a barrier, max / sum reductions of host scalars for timing and throughput,
and a deterministic work-balanced assignment of items to ranks.
"""

from __future__ import annotations

import datetime
import os
from typing import Callable, List, Optional, Sequence, Tuple, TypeVar

Item = TypeVar("Item")


def env_rank() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def setup(backend: str = "nccl", timeout_s: float = 120.0) -> Tuple[int, int, int]:
    """Join the process group when WORLD_SIZE > 1; with NCCL the local GPU is
    made current first.  Returns (world, rank, local rank)."""
    world, rank, local = env_rank()
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def teardown() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()


def _active() -> bool:
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier() -> None:
    if _active():
        import torch.distributed as dist
        dist.barrier()


def _reduce(x: float, op) -> float:
    if not _active():
        return float(x)
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float) -> float:
    """Largest value over the ranks (the job's time is its slowest rank's)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX if _active() else None)


def sum_over_ranks(x: float) -> float:
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM if _active() else None)


def shard(items: Sequence[Item], world: int, rank: int, work: Optional[Callable[[Item], float]] = None) -> List[Item]:
    """This rank's share of ``items``: greedy longest-processing-time
    assignment by ``work`` (largest item to the least loaded rank, ties to
    the lower rank), identical on every rank; order within a share follows
    ``items``.  Without ``work`` every item weighs 1 (round robin)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside world of {world}")
    w = [float(work(it)) if work is not None else 1.0 for it in items]
    order = sorted(range(len(items)), key=lambda k: (-w[k], k))
    load = [0.0] * world
    owner = [0] * len(items)
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += w[k]
    return [it for k, it in enumerate(items) if owner[k] == rank]
