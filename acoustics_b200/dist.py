"""Process-group plumbing for running independent solves on several GPUs.

The FDTD step does not shard: one GPU holds a whole solve (the largest
workload, 384x384x256 cells, needs under 4 GB).  Multi-GPU runs are replicas:
every rank steps its own solves, and the only collective is the
max-over-ranks reduction of the measured time (plus barriers), so the
whole-job throughput is  sum over ranks of work / slowest rank's time.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Optional


@dataclass
class Ranks:
    world: int
    rank: int
    local: int
    pg: Optional[object]   # torch.distributed module when initialised
    device: str            # tensor device of the collectives ("cuda" or "cpu")


def init_from_env(backend: Optional[str] = None, timeout_s: float = 120.0) -> Ranks:
    """Read RANK/LOCAL_RANK/WORLD_SIZE (torchrun) and join the group when WORLD_SIZE > 1."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return Ranks(1, 0, local, None, "cpu")
    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return Ranks(world, rank, local, dist, "cuda" if backend == "nccl" else "cpu")


def max_over_ranks(x: float, r: Ranks) -> float:
    if r.pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=r.device)
    r.pg.all_reduce(t, op=r.pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, r: Ranks) -> float:
    if r.pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=r.device)
    r.pg.all_reduce(t, op=r.pg.ReduceOp.SUM)
    return float(t.item())


def barrier(r: Ranks):
    if r.pg is not None:
        r.pg.barrier()


def weak_scaling_throughput(units_this_rank: float, seconds_this_rank: float, r: Ranks) -> float:
    """Whole-job throughput: all ranks' units divided by the slowest rank's time."""
    total = sum_over_ranks(units_this_rank, r)
    slowest = max_over_ranks(seconds_this_rank, r)
    return total / slowest


def shutdown(r: Ranks):
    if r.pg is not None:
        r.pg.destroy_process_group()
