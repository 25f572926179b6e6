"""One process per GPU: rank bookkeeping for replicas of a solve.

The hot path does not shard across GPUs in this tier (every rank holds a
whole problem), so ranks only meet for timing: a barrier before and after the
timed region and the maximum of the ranks' times.  Works with NCCL (CUDA
tensors) and gloo (CPU tensors).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class RankInfo:
    world: int
    rank: int
    local: int
    backend: str


def init(backend: str = "nccl", timeout_s: int = 300) -> RankInfo:
    """Reads WORLD_SIZE / RANK / LOCAL_RANK (torchrun) and joins the group
    when there is more than one rank."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group(backend,
                                    timeout=datetime.timedelta(seconds=timeout_s))
    return RankInfo(world, rank, local, backend)


def _tensor(v: float, info: RankInfo):
    import torch
    dev = f"cuda:{info.local}" if info.backend == "nccl" else "cpu"
    return torch.tensor([float(v)], dtype=torch.float64, device=dev)


def barrier(info: RankInfo) -> None:
    import torch
    if info.backend == "nccl":
        torch.cuda.synchronize(info.local)
    if info.world > 1:
        import torch.distributed as dist
        t = _tensor(0.0, info)
        dist.all_reduce(t)  # a collective every rank takes in the same order
        if info.backend == "nccl":
            torch.cuda.synchronize(info.local)


def max_over_ranks(v: float, info: RankInfo) -> float:
    if info.world == 1:
        return float(v)
    import torch.distributed as dist
    t = _tensor(v, info)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, seconds: float, info: RankInfo) -> float:
    """Units all ranks processed divided by the slowest rank's time."""
    t = max_over_ranks(seconds, info)
    return info.world * units_per_rank / t


def finalize(info: RankInfo) -> None:
    if info.world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
