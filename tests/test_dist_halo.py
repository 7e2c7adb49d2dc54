"""The z-slab ghost exchange (stx.dist.exchange_z, the MPI half of the
reference's bcswap in z, base_gpu.F90:1132-1196) among two gloo ranks on CPU:
each rank's bottom ghosts receive its lower neighbour's top interior planes and
its top ghosts its upper neighbour's bottom planes, over the interior (i, j)
columns only (periodic over the ranks); the rest of the array is untouched.
With one rank the exchange is the periodic copy within the slab."""
import os
import socket

import numpy as np
import pytest

import helpers as H  # noqa: F401  (puts the package on sys.path)

NG, NZ, NY, NX, NVAR = 3, 5, 4, 6, 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _field(rank):
    import torch
    F = torch.full((NVAR, NZ + 2 * NG, NY + 2 * NG, NX + 2 * NG), float("nan"), dtype=torch.float64)
    m, k, j, i = np.meshgrid(np.arange(NVAR), np.arange(NZ), np.arange(NY), np.arange(NX), indexing="ij")
    F[:, NG:NG + NZ, NG:NG + NY, NG:NG + NX] = torch.from_numpy(1000.0 * rank + 100.0 * m + 10.0 * k + j + 0.01 * i)
    return F


def _check(F, rank, world):
    lo, hi = (rank - 1) % world, (rank + 1) % world
    Flo, Fhi = _field(lo), _field(rank if world == 1 else hi)
    if world == 1:
        Flo = Fhi = _field(rank)
    ij = (slice(NG, NG + NY), slice(NG, NG + NX))
    assert np.array_equal(F[(slice(None), slice(0, NG)) + ij].numpy(), Flo[(slice(None), slice(NZ, NZ + NG)) + ij].numpy())
    assert np.array_equal(F[(slice(None), slice(NZ + NG, NZ + 2 * NG)) + ij].numpy(),
                          Fhi[(slice(None), slice(NG, 2 * NG)) + ij].numpy())
    ref = _field(rank)
    ref[(slice(None), slice(0, NG)) + ij] = F[(slice(None), slice(0, NG)) + ij]
    ref[(slice(None), slice(NZ + NG, NZ + 2 * NG)) + ij] = F[(slice(None), slice(NZ + NG, NZ + 2 * NG)) + ij]
    assert np.array_equal(F.numpy(), ref.numpy(), equal_nan=True)     # nothing else written


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from stx import dist as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        F = _field(rank)
        D.exchange_z(F, NG)
        _check(F, rank, world)
        q.put((rank, "ok"))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_one_rank_exchange_is_the_periodic_copy():
    from stx import dist as D
    F = _field(0)
    D.exchange_z(F, NG)
    _check(F, 0, 1)


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchange_z_ghosts(world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {r: "ok" for r in range(world)}, res
