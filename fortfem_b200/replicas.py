"""Several GPUs on independent systems: one process per GPU, no collective on
the data path.

The benchmarked workloads shard without any exchange: the single-system
benchmark solves one replica of the system per GPU, and a serving stream is
a set of independent requests.  What crosses processes is bookkeeping only:
which rank serves which request, the slowest rank's time, and the latencies
gathered for the report.  Ranks use torch.distributed (NCCL on GPUs, gloo on
the CPU for tests) for that bookkeeping; every rank calls the collectives
below in the same order.
"""
from __future__ import annotations

import os
from typing import List, Sequence

from .serving import Request, free_dofs


def env():
    """(rank, world size, local rank) of this process, from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def partition_requests(requests: Sequence[Request], world: int) -> List[List[Request]]:
    """Split a request stream across `world` GPUs, each request (in arrival
    order) to the rank with the least estimated work so far (free DoFs as the
    work estimate; ties to the lower rank).  Deterministic, so every rank
    computes the same split without communicating."""
    shares: List[List[Request]] = [[] for _ in range(world)]
    load = [0] * world
    for r in sorted(requests, key=lambda q: (q.arrival, q.rid)):
        k = min(range(world), key=lambda i: (load[i], i))
        shares[k].append(r)
        load[k] += free_dofs(r.key)
    return shares


def _device_for(backend: str):
    import torch
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float) -> float:
    """The largest `value` over all ranks (the job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=_device_for(dist.get_backend()))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=_device_for(dist.get_backend()))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_lists(local: list) -> list:
    """Concatenation of every rank's `local` list, in rank order, on all ranks."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(local))
    return [x for part in out for x in part]
