"""Multi-GPU plumbing: one process per GPU, iterations sharded round-robin.

UPBP iterations are independent given (seed, iteration): the radius schedule
and the random streams are pure functions of the iteration index, so rank r
of N renders iterations r, r+N, r+2N, ... with its own light pass and photon
maps, and the images are combined once, at output time, by a sum-reduction
of the per-rank accumulations (NCCL all-reduce over NVLink on B200; gloo in
the CPU tests).  There is no exchange inside an iteration.
"""
from __future__ import annotations

import numpy as np


def shard_iterations(rank: int, world: int, total: int, start: int = 0) -> list[int]:
    """Iterations rank `rank` of `world` renders out of [start, start + total)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("invalid rank/world")
    return list(range(start + rank, start + total, world))


def combine(accumulated_sum: np.ndarray, iterations_done: int, group=None, device=None):
    """Sum-reduces per-rank (sum of iteration images, iteration count) and
    returns the average image over all ranks' iterations."""
    import torch
    import torch.distributed as dist

    t = torch.as_tensor(np.ascontiguousarray(accumulated_sum, np.float64), device=device)
    n = torch.tensor([float(iterations_done)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, group=group)
        dist.all_reduce(n, group=group)
    return (t / n).cpu().numpy()
