"""Multi-process plumbing for running independent signals on several GPUs.

The transform path has no exchange step across signals, so ranks are
replicas: each rank owns a contiguous share of the signal indices, runs them
on its own GPU, and only timing is combined (max over ranks).  One process
per GPU; torch.distributed with NCCL on GPUs, gloo on CPU (tests).
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass
class RankInfo:
    rank: int
    world: int
    local: int


def rank_info() -> RankInfo:
    """RANK / WORLD_SIZE / LOCAL_RANK as set by torch.distributed.run."""
    return RankInfo(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_total: int, rank: int, world: int) -> range:
    """Contiguous share of signal indices [0, n_total) for `rank`; shares differ
    in size by at most one and cover every index exactly once."""
    base, extra = divmod(n_total, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def signal_seed(base: int, rank: int, index: int) -> int:
    """Seed of signal `index` on `rank` (distinct across ranks and indices)."""
    return base + 1_000_003 * rank + index


def init(backend: str | None = None, timeout_s: int = 120):
    """Initialises the process group when WORLD_SIZE > 1 (no-op otherwise)."""
    import datetime

    import torch.distributed as dist
    info = rank_info()
    if info.world > 1 and not dist.is_initialized():
        if backend is None:
            import torch
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return info


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (elapsed time) over all ranks."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_throughput(units_done_total: float, max_seconds: float) -> float:
    """Whole-job units per second: all ranks' units over the slowest rank's time."""
    return units_done_total / max_seconds if max_seconds > 0 else float("nan")


def barrier():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.barrier()


def finalize():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
