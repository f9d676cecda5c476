"""Multi-GPU replicas of the batched clustering workload.

Events are independent, so N GPUs run N replicas: one process per GPU (the
launcher sets RANK / LOCAL_RANK / WORLD_SIZE), each clustering its own shard
of events with no data exchanged. The only collectives are host-side
bookkeeping: a barrier around the timed region and the maximum of the per-rank
device times; throughput is the points of all ranks over that maximum.
`torch.distributed` carries them over NCCL between GPUs, or over gloo where no
GPU is present (the multi-rank tests run that way on CPU).
"""

from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass(frozen=True)
class Ranks:
    world: int
    rank: int
    local: int


def from_env() -> Ranks:
    """Rank layout the launcher exported (a single rank when absent)."""
    return Ranks(world=int(os.environ.get("WORLD_SIZE", "1")),
                 rank=int(os.environ.get("RANK", "0")),
                 local=int(os.environ.get("LOCAL_RANK", "0")))


def init(r: Ranks, backend: str | None = None, timeout_s: float = 300.0) -> str | None:
    """Joins the process group when world > 1; returns the backend in use."""
    if r.world == 1:
        return None
    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(r.local)
        kw["device_id"] = torch.device("cuda", r.local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return backend


def finish(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def barrier(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(x: float, r: Ranks, op) -> float:
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, r: Ranks) -> float:
    """Largest value over all ranks (the job's time is its slowest rank's)."""
    if r.world == 1:
        return float(x)
    import torch.distributed as dist
    return _reduce(x, r, dist.ReduceOp.MAX)


def sum_over_ranks(x: float, r: Ranks) -> float:
    if r.world == 1:
        return float(x)
    import torch.distributed as dist
    return _reduce(x, r, dist.ReduceOp.SUM)


def event_seed(rank: int, base: int = 3) -> int:
    """Seed of rank `rank`'s shard of the batch workload (distinct per rank)."""
    return base + 1000 * rank


def job_throughput(points_all_ranks: float, ms_max: float) -> float:
    """Points per second of the whole job: all ranks' points over the slowest rank's time."""
    return points_all_ranks / (ms_max * 1e-3)
