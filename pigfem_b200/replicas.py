"""Replica runs on several GPUs of one node: one process per GPU, each with its own independent
work (its own RVE, batch or request stream, seeded by rank), no collective on the data path.
The only communication is the barrier around a timed region and the maximum of the timings over
ranks, so a run's throughput is (units on all ranks) / (slowest rank's time).

The helpers take the backend the caller picked: NCCL with one GPU per rank in bench.py, gloo on
CPU in the tests.
"""
from __future__ import annotations

import datetime
import os
from typing import List, Sequence


def dist_env():
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, local_rank: int = 0, timeout_s: float = 120.0) -> bool:
    """Joins the process group when the world has more than one rank; returns whether it did.
    The short timeout makes ranks that wait for a missing peer end with an error."""
    ws, _, _ = dist_env()
    if ws <= 1:
        return False
    import torch
    import torch.distributed as dist
    kw = {}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return True


def _active() -> bool:
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier():
    if _active():
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(values: Sequence[float], device: str = "cpu") -> List[float]:
    """Element-wise maximum over ranks (the slowest rank's timings); the values themselves when
    there is one rank.  `device` is where the reduction runs: "cuda" for NCCL, "cpu" for gloo."""
    vals = [float(v) for v in values]
    if not _active():
        return vals
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu().tolist()]


def sum_over_ranks(values: Sequence[float], device: str = "cpu") -> List[float]:
    """Element-wise sum over ranks (whole-job totals of per-rank counts and rates)."""
    vals = [float(v) for v in values]
    if not _active():
        return vals
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.cpu().tolist()]


def aggregate_rate(units_per_rank: float, world_size: int, total_ms: float) -> float:
    """Whole-job throughput: every rank processed units_per_rank in at most total_ms."""
    return world_size * units_per_rank / (total_ms * 1e-3)


def finish():
    """Leaves the process group (after a final barrier)."""
    if _active():
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
