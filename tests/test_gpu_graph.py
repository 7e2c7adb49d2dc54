"""Captured steps (stx_graph_*): nsteps iterations of the integration loop
replayed from one CUDA graph give the same fields, bit for bit, as the same
steps called one by one, for the 1-D flame ("simpler" splitting, ROK4) and the
shock tube (Strang, ROK4), and the time seen by the chemistry advances.  With a
CFL-driven step (stx_graph_create_cfl) the graph also forms every step's dt on
the device from the CFL maxima: the same dt sequence, time and fields as the
host loop that reads the maxima back every step, for the 1-D shock tube of
config 1, the flame with the simpler splitting and a 3-D turbulence box."""
import numpy as np
import pytest
import torch

import helpers as H  # noqa: F401  (puts the package on sys.path)

pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from stx import configs  # noqa: E402
from stx.solver import Solver  # noqa: E402


def _eager_vs_graph(make_case, nsteps, per_graph):
    a = Solver(make_case())
    a.prepare()
    dts = []
    for _ in range(nsteps):
        a.step()
        dts.append(a.dt)
    b = Solver(make_case())
    b.prepare()
    g = b.capture(per_graph)
    gdts = []
    for _ in range(nsteps // per_graph):
        b.replay(g)
        gdts.append(b.dt)
    torch.cuda.synchronize()
    assert a.time == b.time and a.icyc == b.icyc
    assert gdts == dts[per_graph - 1::per_graph]
    wa, wb = a.host_w(), b.host_w()
    assert np.isfinite(wa).all()
    assert np.array_equal(wa, wb)
    assert np.array_equal(a.host_w_aux(), b.host_w_aux())
    assert a.status() == b.status()
    a.close()
    b.close()
    return dts


def test_graph_flame_simpler_splitting():
    _eager_vs_graph(lambda: configs.flame_case(400, phi=0.9, Tu=400.0), 6, 3)


def test_graph_shock_tube_strang():
    _eager_vs_graph(lambda: configs.tube_case(300, 1), 8, 4)


def test_graph_cfl_shock_tube_config1():
    dts = _eager_vs_graph(lambda: configs.config1_case(600, cfl=0.5), 12, 4)
    assert len(set(dts)) > 1              # the step size does change from step to step


def test_graph_cfl_flame_simpler_splitting():
    def case():
        c = configs.flame_case(400, phi=0.9, Tu=400.0)
        c.cfl = 0.4
        return c
    _eager_vs_graph(case, 6, 3)


def test_graph_cfl_turbulence_3d():
    def case():
        c = configs.turbulence_case(16, alloc_fields=True)
        c.w[:], c.w_aux[:] = configs.turbulence_fields(c, 7)
        return c
    _eager_vs_graph(case, 4, 2)


def test_graph_refuses_dt_recompute_interval():
    case = configs.turbulence_case(8, alloc_fields=True)
    case.iter_dt_recompute = 2
    s = Solver(case)
    with pytest.raises(ValueError):
        s.capture(2)
    s.close()
