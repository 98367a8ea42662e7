"""Multi-GPU plumbing: one process per GPU, independent SCFT instances.

A single instance (at most ~17 MB per field at the benchmark sizes) does not
shard usefully, so several GPUs run replicas or disjoint subsets of a batch of
instances; the only collectives are a barrier and scalar reductions (max of the
per-rank device times, sums of counts).  NCCL carries them between GPUs, gloo on
CPU-only hosts.
"""
from __future__ import annotations

import datetime
import heapq
import os


def dist_env():
    """(rank, world_size, local_rank) from the torchrun environment (defaults: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: float = 120.0, device=None):
    """Initialise the default process group when world_size > 1; returns torch.distributed or None."""
    rank, world, local = dist_env()
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist

    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        kw["device_id"] = device if device is not None else torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return dist


def _device_for(dist):
    import torch

    if dist is not None and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, x: float) -> float:
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, x: float) -> float:
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard_instances(costs, world: int):
    """Split instances (cost per instance, e.g. space_size_phy x contour steps) over
    `world` ranks: longest-processing-time-first greedy, deterministic.  Returns one
    sorted list of instance indices per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in out]
