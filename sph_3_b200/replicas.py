"""Multi-GPU execution of this path: independent replicas.

The SPH + gravity step of one particle system has no exchange step that this
build distributes (a single system stays on one GPU); several GPUs each step
their own system (or their own share of a batched ensemble), so the only
cross-rank operations are timing and result reductions.  They work with the
"nccl" backend on GPUs and with "gloo" on CPU (used by the tests).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def world():
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def _device_for_backend():
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """max of a per-rank scalar (e.g. a timed region in ms) over all ranks."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units_this_rank: float, seconds_this_rank: float) -> float:
    """units processed by all ranks / the slowest rank's time."""
    return sum_over_ranks(units_this_rank) / max_over_ranks(seconds_this_rank)


def shard_clouds(counts, rank, nranks):
    """Contiguous share of a batched ensemble's clouds for one rank (balanced
    by particle count); returns (first cloud, last cloud + 1)."""
    import numpy as np
    c = np.asarray(counts, dtype=np.int64)
    cum = np.concatenate([[0], np.cumsum(c)])
    total = cum[-1]
    lo = int(np.searchsorted(cum, total * rank / nranks, side="left"))
    hi = int(np.searchsorted(cum, total * (rank + 1) / nranks, side="left"))
    if rank == nranks - 1:
        hi = len(c)
    return min(lo, len(c)), min(hi, len(c))
