"""The continuous-batching request loop (stx/serve.py): a mix of 0-D reactor,
1-D flame and 2-D shock-tube requests that arrive while others run; every
result equals the same request served alone (bit for bit), and the loop
reports throughput and p50/p99 latency."""
import numpy as np
import pytest
import torch

import helpers as H  # noqa: F401  (puts the package on sys.path)

pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from stx import configs  # noqa: E402
from stx.reactors import sample_h2air  # noqa: E402
from stx.serve import Request, Server  # noqa: E402


def _mix():
    mech = configs.mechanism("h2air_9sp")
    T0, p0, Y0 = sample_h2air(10, 4, mech, T_range=(1200.0, 1500.0))
    reqs = [Request(i, "reactor", 0.004 * i, {"T0": float(T0[i]), "p0": float(p0[i]), "Y0": Y0[:, i].copy()})
            for i in range(10)]
    reqs += [Request(10, "flame1d", 0.001, {"nx": 384, "phi": 0.8, "Tu": 400.0}, steps=6),
             Request(11, "flame1d", 0.003, {"nx": 256, "phi": 1.2, "Tu": 600.0}, steps=5),
             Request(12, "tube2d", 0.002, {"nx": 128, "ny": 8}, steps=4),
             Request(13, "flame1d", 0.020, {"nx": 512, "phi": 0.6, "Tu": 300.0}, steps=3)]
    return reqs


def _same(a, b):
    assert a.kind == b.kind
    for k, v in a.result.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, b.result[k]), (a.rid, k)
        else:
            assert v == b.result[k], (a.rid, k)


def test_served_mix_equals_each_request_alone():
    srv = Server(max_grid=3, chunk=2, t_max=5e-3, max_steps=60000)
    try:
        mix = _mix()
        stats = srv.run(mix, realtime=True)
        assert stats["requests"] == len(mix)
        assert all(r.done is not None and r.latency > 0 for r in mix)
        assert 0 < stats["p50_s"] <= stats["p99_s"]
        assert stats["max_grid_in_flight"] >= 2          # grid solves overlapped on the device
        for r in mix:
            alone = _mix()[r.rid]
            srv.run([alone], realtime=False)
            _same(r, alone)
        for r in mix:
            if r.kind == "reactor":
                assert r.result["t_ign"] > 0
            else:
                assert np.isfinite(r.result["w"]).all() and r.result["status"] & ~0x1 == 0
    finally:
        srv.close()


def test_memory_budget_limits_admission():
    """With a budget that fits one grid solve, grid solves run one at a time."""
    srv = Server(max_grid=8, chunk=2, t_max=5e-3, mem_budget=1)
    try:
        reqs = [Request(i, "flame1d", 0.0, {"nx": 256, "phi": 1.0, "Tu": 500.0}, steps=2) for i in range(3)]
        stats = srv.run(reqs, realtime=False)
        assert stats["max_grid_in_flight"] == 1
        assert all(r.done is not None for r in reqs)
        for r in reqs[1:]:
            assert np.array_equal(r.result["w"], reqs[0].result["w"])
    finally:
        srv.close()


def test_context_on_shared_tables_equals_a_fresh_one():
    """stx_ctx_create_like: a solver on another solver's device tables gives the
    same fields, bit for bit, as one that uploaded its own."""
    from stx import mech as M
    from stx.solver import Solver
    tb = M.build_tables(configs.mechanism("h2air_9sp"), 101325.0, 200.0, 5500.0, 1.0)
    base = Solver(configs.flame_case(64, tables=tb, mech_name="h2air_9sp"))
    make = lambda: configs.flame_case(300, phi=0.9, Tu=450.0, tables=tb, mech_name="h2air_9sp")
    out = []
    for kw in ({}, {"tables_from": base}):
        s = Solver(make(), **kw)
        s.prepare()
        for _ in range(3):
            s.step()
        out.append(s.host_w())
        s.close()
    base.close()
    assert np.array_equal(out[0], out[1])
