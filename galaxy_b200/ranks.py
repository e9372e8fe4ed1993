"""One process per GPU: rank discovery, sharding of independent systems, and the
reductions of the timing contract.

A single system's step does not shard (every target walks the whole tree), so more
GPUs run more systems: replicas of one workload, or a partition of many independent
systems. There is no data-path collective; the only collectives are the barrier
around the timed region and the max / sum of the per-rank results. Launch under
``torchrun`` (RANK / WORLD_SIZE / LOCAL_RANK / MASTER_* from the environment); NCCL
when CUDA is present, gloo otherwise.
"""

from __future__ import annotations

import heapq
import os
from datetime import timedelta


def env() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the torchrun environment (0, 1, 0 alone)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(timeout_s: float = 300.0):
    """Join the process group when WORLD_SIZE > 1; returns (dist or None, rank, world, local)."""
    rank, world, local = env()
    if world <= 1:
        return None, 0, 1, 0
    import torch
    import torch.distributed as dist

    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return dist, rank, world, local


def _device(local: int):
    import torch

    return torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")


def barrier(dist, local: int) -> None:
    if dist is None:
        return
    import torch

    if torch.cuda.is_available():
        dist.barrier(device_ids=[local])
    else:
        dist.barrier()


def _reduce(dist, v: float, local: int, op_name: str) -> float:
    if dist is None:
        return float(v)
    import torch

    t = torch.tensor([float(v)], dtype=torch.float64, device=_device(local))
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(dist, v: float, local: int = 0) -> float:
    """The slowest rank's time: the timed region ends when every rank has finished."""
    return _reduce(dist, v, local, "MAX")


def sum_over_ranks(dist, v: float, local: int = 0) -> float:
    return _reduce(dist, v, local, "SUM")


def shard(sizes, world: int) -> list[list[int]]:
    """Partition systems (given by particle count) across `world` ranks: largest first,
    each to the rank with the fewest particles so far (ties to the lower rank). Every
    index lands on exactly one rank; each rank's list is in ascending index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(x) for x in out]
