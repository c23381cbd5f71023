"""Multi-process plumbing for running independent simulations on several GPUs.

A single PM simulation does not split into independent pieces, so multi-GPU runs are
replicas: every rank runs its own simulations (its share of the requests), nothing is
exchanged on the data path, and timings are reduced as the max over ranks. One process per
GPU, launched by torch.distributed.run; NCCL on GPUs, gloo for CPU tests.
"""

from __future__ import annotations

import datetime
import os

import torch


def world_from_env():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(
        os.environ.get("LOCAL_RANK", "0"))


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """Initialise the process group when WORLD_SIZE > 1; returns (world, rank, local_rank)."""
    world, rank, local = world_from_env()
    if world > 1 and not torch.distributed.is_initialized():
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    elif backend == "nccl" and torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier():
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.barrier()
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of a scalar over all ranks (the job's time is its slowest rank's)."""
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(value)
    dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(value)
    dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
    return float(t.item())


def shard(items, world: int, rank: int):
    """The items rank `rank` owns: round-robin, so every rank gets a near-equal share."""
    return list(items)[rank::world]


def finalize():
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.destroy_process_group()
