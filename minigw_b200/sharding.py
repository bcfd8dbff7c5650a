"""Frequency sharding of one G0W0 solve over ranks (one GPU per rank).

Each rank solves the screened interaction for a contiguous shard of the integration frequencies
f' (every W_c(i w_f') is solved exactly once, on one rank) and contracts it onto the whole output
grid; one all-reduce (SUM) of the nmo x nfreq complex partial Sigma_c then gives every rank the
full Sigma_c.  This replaces the reference's MPI distribution of output frequencies
(src/gw/sigma_c_driver.cpp:368-401 with mpi_allreduce_sum_in_place, src/mpi_context.cpp:45-64),
which solves every W_c on every rank.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def shard_bounds(nfreq: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced split of range(nfreq): shard sizes differ by at most one."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(nfreq, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def sharded_sigma_c(partial: Callable[[int, int], np.ndarray], nfreq: int, world: int, rank: int,
                    allreduce_sum: Callable[[np.ndarray], np.ndarray]) -> np.ndarray:
    """Full Sigma_c on every rank: `partial(f_begin, f_end)` returns this rank's nmo x nfreq complex
    partial sum (e.g. B200Backend.sigma_c_shard), `allreduce_sum` sums a float64 array over ranks."""
    b, e = shard_bounds(nfreq, world, rank)
    part = np.ascontiguousarray(partial(b, e), dtype=np.complex128)
    summed = allreduce_sum(part.view(np.float64).copy())
    return np.ascontiguousarray(summed).view(np.complex128).reshape(part.shape)


def torch_allreduce_sum(device: str | None = None) -> Callable[[np.ndarray], np.ndarray]:
    """An allreduce_sum over the default torch.distributed group (NCCL: device = 'cuda:N'; gloo: None)."""
    import torch
    import torch.distributed as dist

    def reduce(a: np.ndarray) -> np.ndarray:
        t = torch.from_numpy(a)
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t.cpu().numpy()

    return reduce
