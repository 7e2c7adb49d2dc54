"""Multi-rank host logic on CPU: two gloo ranks, each with its own box, agree on
the global dt (max-reduction of the CFL maxima, multideal_gpu.F90:1644-1654) and
on the slowest-rank timing, exactly as the NCCL path of bench.py does on GPUs."""
import os
import socket

import numpy as np
import pytest

import helpers as H


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import ctypes as C
    import sys
    sys.path.insert(0, os.path.join(H.REPO, "tests"))
    import torch.distributed as dist
    import helpers as HH
    from driver import OracleSolver
    from stx import dist as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = HH.synthetic_case(n=(8, 6, 5), seed=100 + rank, amp_u=40.0 + 40.0 * rank)
        o = OracleSolver(case, threads=1)
        o.update_ghost(1)
        o.compute_aux(1, 1)
        out = (C.c_double * 9)()
        o.lib.ox_compute_dt(o.ctx, C.c_void_p(o.w_aux.ctypes.data), None, out)
        local = list(out)
        dt = D.global_dt(local, 0.5)
        slow = D.max_over_ranks(1.0 + rank)
        fixed = D.global_dt(local, -2e-8)
        q.put((rank, local, dt, slow, fixed))
        o.close()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_global_dt():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    all_max = max(max(r[1]) for r in res)
    for rank, local, dt, slow, fixed in res:
        assert dt == 0.5 / all_max
        assert slow == 2.0
        assert fixed == 2e-8
    # the two boxes differ, so the reduction mattered for one of them
    assert max(res[0][1]) != max(res[1][1])
