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


# ---------------------------------------------------------------- z-slab halos
STX_BC_EXCHANGE = -1     # include/stx.h: a face whose ghosts the caller fills


def exchange_z(F: torch.Tensor, ng: int, group=None):
    """Fill the z ghost layers of the ghosted fields F (nvar, nzg, nyg, nxg)
    from the neighbouring z slabs of a periodic z-slab decomposition over the
    ranks of group: rank r's bottom ghosts take rank r-1's top ng interior
    planes, its top ghosts rank r+1's bottom ones (the MPI sendrecv of the
    reference's bcswap in z, base_gpu.F90:1132-1196).  As the periodic swap
    does, only the interior (i, j) columns of the ghost planes are written.
    One rank: the periodic copy within the slab.  Several: one grouped
    isend/irecv exchange (NCCL on GPUs, gloo on CPU), on the current stream."""
    import torch.distributed as dist
    nzg, nyg, nxg = F.shape[1:]
    nz, ny, nx = nzg - 2 * ng, nyg - 2 * ng, nxg - 2 * ng
    ij = (slice(ng, ng + ny), slice(ng, ng + nx))
    lo_in, hi_in = (slice(None), slice(ng, 2 * ng)) + ij, (slice(None), slice(nz, nz + ng)) + ij
    lo_gh, hi_gh = (slice(None), slice(0, ng)) + ij, (slice(None), slice(nz + ng, nz + 2 * ng)) + ij
    ws = dist.get_world_size(group) if (dist.is_available() and dist.is_initialized()) else 1
    if ws == 1:
        top, bot = F[hi_in].clone(), F[lo_in].clone()
        F[lo_gh] = top
        F[hi_gh] = bot
        return
    rank = dist.get_rank(group)
    up, down = (rank + 1) % ws, (rank - 1) % ws
    gup = dist.get_global_rank(group, up) if group is not None else up
    gdown = dist.get_global_rank(group, down) if group is not None else down
    send_up, send_dn = F[hi_in].contiguous(), F[lo_in].contiguous()
    recv_dn, recv_up = torch.empty_like(send_up), torch.empty_like(send_dn)
    # the same order on every rank: with two ranks both messages go to the same
    # peer and are matched in posting order (top -> peer's bottom first)
    ops = [dist.P2POp(dist.isend, send_up, gup, group), dist.P2POp(dist.irecv, recv_dn, gdown, group),
           dist.P2POp(dist.isend, send_dn, gdown, group), dist.P2POp(dist.irecv, recv_up, gup, group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    F[lo_gh] = recv_dn
    F[hi_gh] = recv_up


def make_z_slab(case):
    """Turn a case's z faces into exchange interfaces (STX_BC_EXCHANGE): the
    rank's box becomes one z slab of a periodic decomposition whose ghosts
    exchange_z fills."""
    case.bctags[4] = case.bctags[5] = STX_BC_EXCHANGE
    case.periodic[2] = False
    return case


class ZSlabExchange:
    """The stx_set_exchange callback of a Solver on a z-slab case: every
    periodic swap of the library (conserved variables, Ducros sensor, div/3)
    is followed by exchange_z on the swapped fields."""

    def __init__(self, solver, group=None):
        import ctypes as C
        from .native import EXCHANGE_FN
        self.sol, self.group, self.ng = solver, group, solver.case.ng
        self._fn = EXCHANGE_FN(self._call)          # kept alive with the object
        self.error = None

    def _field(self, ptr: int, nvar: int) -> torch.Tensor:
        s = self.sol
        base = s.w_aux if s.w_aux.data_ptr() <= ptr < s.w_aux.data_ptr() + s.w_aux.numel() * 8 else s.w
        first = (ptr - base.data_ptr()) // (8 * base[0].numel())
        return base[first:first + nvar]

    def _call(self, user, stream, field, nvar):
        try:
            exchange_z(self._field(int(field), int(nvar)), self.ng, self.group)
            return 0
        except Exception as e:          # reported through the library's return code
            self.error = e
            return -2

    def install(self):
        import ctypes as C
        from .native import check
        check(self.sol.lib.stx_set_exchange(self.sol.ctx, self._fn, None), "stx_set_exchange")
        return self
