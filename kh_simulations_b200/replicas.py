"""Replica plumbing for running independent Kelvin–Helmholtz runs on several
GPUs of one node.

The step does not shard across GPUs: each rank advances its own run (the
same configuration), with no collective on the data path.  The only
cross-rank traffic is timing: a barrier on each side of the timed region
and the maximum of the per-rank device times, from which the whole-job
throughput is the units all ranks processed divided by that maximum.

The reference has no multi-GPU form (ymgpu2d/main_ym.cu runs one GPU per
process; campaigns launch one process per configuration, ymgpu2d/scripts/).

Works with the ``nccl`` backend (one process per GPU, CUDA tensors) and
with ``gloo`` (CPU tensors), which is how the multi-process logic is tested
without GPUs.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    world: int
    rank: int
    local: int
    backend: str | None  # None when world == 1 (no process group)


def init(backend: str = "nccl", timeout_s: float = 600.0) -> Ranks:
    """Reads RANK / LOCAL_RANK / WORLD_SIZE (torchrun) and, for more than one
    rank, joins the process group.  With nccl the rank's GPU is LOCAL_RANK."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return Ranks(1, 0, 0, None)
    import torch
    import torch.distributed as dist

    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device(f"cuda:{local}")
    dist.init_process_group(backend, **kw)
    return Ranks(world, rank, local, backend)


def _device(r: Ranks):
    import torch

    return torch.device(f"cuda:{r.local}") if r.backend == "nccl" else torch.device("cpu")


def barrier(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, r: Ranks) -> float:
    """The largest of the ranks' values (every rank gets it)."""
    if r.world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(r))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, ms_max: float, r: Ranks) -> float:
    """Whole-job throughput: units every rank processed (weak scaling: each
    rank does the same work) over the slowest rank's time."""
    return units_per_rank * r.world / (ms_max / 1e3)


def finish(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
