"""Multi-rank plumbing of the reacting step (one process per GPU).

The reference decomposes the domain over MPI ranks and reduces the nine CFL
maxima of compute_dt_cuf with mpi_allreduce(MPI_MAX) before forming dt
(src/multideal/multideal_gpu.F90:1644-1654).  Here torch.distributed carries
the same reduction: NCCL on GPUs, gloo on CPU ranks (tests).
"""
from __future__ import annotations

from typing import Sequence

import torch


def world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def global_dt(local9: Sequence[float], cfl: float, device=None) -> float:
    """dt = cfl / max over ranks and over the nine inverse time scales
    (convective, viscous, conductive in x, y, z); cfl < 0 means a fixed -cfl."""
    if cfl < 0:
        return -cfl
    import torch.distributed as dist
    m = torch.tensor([float(v) for v in local9], dtype=torch.float64, device=device)
    ws, _ = world()
    if ws > 1:
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return cfl / float(m.max())


def max_over_ranks(value: float, device=None) -> float:
    """Max of a scalar over ranks (timings are reported as the slowest rank)."""
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    ws, _ = world()
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
