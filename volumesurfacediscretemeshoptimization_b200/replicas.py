"""Replicas on several GPUs, one process per GPU.

The DMO path has no exchange step: a colour class reads and writes only its own mesh, and the
reference optimises one mesh per process. Several GPUs therefore run independent replicas
(each rank its own seeded mesh: weak scaling), and the only collectives are the barriers around
a timed region and the maximum of the ranks' times, from which the whole-job rate is the units
all ranks processed divided by the slowest rank's time. This module holds that host logic; it
runs over NCCL on GPUs and over gloo on CPU (the multi-process tests).
"""
from __future__ import annotations

import datetime
import os


def rank_info():
    """(rank, world size, local rank) from the launcher's environment (1 process: 0, 1, 0)."""
    r = int(os.environ.get("RANK", "0"))
    w = int(os.environ.get("WORLD_SIZE", "1"))
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    return r, w, lr


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """Joins the process group when the world has more than one rank; returns
    torch.distributed, or None for a single process. The short timeout turns a rank that
    never arrives into an error on the others instead of a hang."""
    _, world, _ = rank_info()
    if world <= 1:
        return None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def replica_seed(rank: int) -> int:
    """Seed of rank r's replica mesh: every rank optimises a different jittered mesh of the
    same size."""
    return int(rank)


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest value over all ranks (the job's time is its slowest rank's)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, ms_max: float, world: int) -> float:
    """Units per second of the whole job: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / (ms_max / 1e3)


def finish(dist) -> None:
    if dist is not None:
        dist.destroy_process_group()
