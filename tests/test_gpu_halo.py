"""The ghost-exchange hook (stx_set_exchange, STX_BC_EXCHANGE faces) on one
GPU: a turbulence box whose z faces are exchange interfaces, filled by
stx.dist.ZSlabExchange (one rank: the periodic copy), advances bit for bit as
the same box with periodic z faces -- the library calls the exchange after
every periodic swap of the step (conserved variables, Ducros sensor, div/3).
A context with an exchange refuses stream capture."""
import numpy as np
import pytest
import torch

import helpers as H  # noqa: F401  (puts the package on sys.path)

pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from stx import configs  # noqa: E402
from stx import dist as D  # noqa: E402
from stx.solver import Solver  # noqa: E402


def _run(slab: bool, steps: int):
    case = configs.turbulence_case(16, alloc_fields=True)
    W, WA = configs.turbulence_fields(case, 11)
    if slab:
        D.make_z_slab(case)
    s = Solver(case, w=torch.from_numpy(W).cuda(), w_aux=torch.from_numpy(WA).cuda())
    x = D.ZSlabExchange(s).install() if slab else None
    s.prepare()
    for _ in range(steps):
        s.step()
    torch.cuda.synchronize()
    assert x is None or x.error is None
    out = case.interior(s.host_w()), case.interior(s.host_w_aux())
    s.close()
    return out


def test_exchange_hook_equals_periodic_faces():
    w0, wa0 = _run(False, 2)
    w1, wa1 = _run(True, 2)
    assert np.array_equal(w0, w1)
    assert np.array_equal(wa0, wa1)


def test_exchange_context_is_not_capturable():
    case = D.make_z_slab(configs.turbulence_case(8, alloc_fields=True, cfl=-1e-9))
    s = Solver(case)
    D.ZSlabExchange(s).install()
    with pytest.raises(RuntimeError):
        s.capture(2)
    s.close()
