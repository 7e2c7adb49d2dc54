"""Captured steps (stx_graph_*): nsteps iterations of the integration loop
replayed from one CUDA graph give the same fields, bit for bit, as the same
steps called one by one, for the 1-D flame ("simpler" splitting, ROK4) and the
shock tube (Strang, ROK4), and the time seen by the chemistry advances."""
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
    for _ in range(nsteps):
        a.step()
    b = Solver(make_case())
    b.prepare()
    g = b.capture(per_graph)
    for _ in range(nsteps // per_graph):
        b.replay(g)
    torch.cuda.synchronize()
    assert a.time == b.time and a.icyc == b.icyc
    wa, wb = a.host_w(), b.host_w()
    assert np.isfinite(wa).all()
    assert np.array_equal(wa, wb)
    assert np.array_equal(a.host_w_aux(), b.host_w_aux())
    assert a.status() == b.status()
    a.close()
    b.close()


def test_graph_flame_simpler_splitting():
    _eager_vs_graph(lambda: configs.flame_case(400, phi=0.9, Tu=400.0), 6, 3)


def test_graph_shock_tube_strang():
    _eager_vs_graph(lambda: configs.tube_case(300, 1), 8, 4)


def test_graph_refuses_cfl_driven_runs():
    case = configs.turbulence_case(8, alloc_fields=True)
    s = Solver(case)
    with pytest.raises(ValueError):
        s.capture(2)
    s.close()
