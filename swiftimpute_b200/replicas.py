"""Sample-sharded replicas: one process per GPU.

Target chains are independent, so several GPUs serve one job by each holding
its own copy of the panel and PBWT index and imputing its own share of the
targets; nothing crosses between ranks while they impute. The only
communication is host-side bookkeeping through torch.distributed (NCCL
between GPUs, gloo on CPU): the slowest rank's time, and an optional gather of
the outputs at rank 0. This stands in for the reference's MultiGPUImputer
(src/api/imputer.hpp:298-328), which is declared but does not split work.
"""
from __future__ import annotations

import numpy as np


def shard(n: int, world: int, rank: int) -> tuple[int, int]:
    """Rows [start, stop) of rank ``rank`` among ``world``: contiguous, sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest ``value`` of all ranks (a step's time is its slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(local: np.ndarray, dist=None) -> np.ndarray | None:
    """Concatenate every rank's rows in rank order at rank 0 (None elsewhere).

    Host arrays through the process group's object gather: meant for results
    that fit in host memory, after the imputation itself is done."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(local, parts, dst=0)
    return np.concatenate(parts, axis=0) if dist.get_rank() == 0 else None
