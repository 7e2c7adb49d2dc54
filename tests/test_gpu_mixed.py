"""The mixed-precision form (stx_set_precision(STX_PREC_MIXED)): central face
fluxes, viscous/diffusive fluxes and transport properties in FP32, the RK
residual, Newton T(e) and chemistry in FP64.  Its error against the FP64 oracle
after whole reacting steps on the turbulence workload must stay within 1e-4
relative in T and in every Y_k > 1e-8 (1e-12 absolute below); the FP64 form on
the same inputs stays within 1e-7."""
import numpy as np
import pytest
import torch

import helpers as H  # noqa: F401  (puts the package on sys.path)

pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from driver import OracleSolver  # noqa: E402
from stx import configs  # noqa: E402
from stx.solver import Solver  # noqa: E402


def _run(case, W, WA, form, steps):
    s = Solver(case, w=torch.from_numpy(W).cuda(), w_aux=torch.from_numpy(WA).cuda())
    s.set_precision(form)
    s.prepare()
    for _ in range(steps):
        s.step()
    torch.cuda.synchronize()
    out = s.host_w(), s.host_w_aux()
    s.close()
    return out


def _errors(case, w, wa, wo, wao):
    ns = case.ns
    T, To = case.interior(wa[case.J("T")]), case.interior(wao[case.J("T")])
    eT = np.max(np.abs(T - To) / To)
    Y, Yo = case.interior(wa[:ns]), case.interior(wao[:ns])
    big = Yo > 1e-8
    eY = np.max(np.abs(Y - Yo)[big] / Yo[big])
    eYs = np.max(np.abs(Y - Yo)[~big]) if (~big).any() else 0.0
    return eT, eY, eYs


def test_mixed_form_within_1e4_of_fp64_oracle():
    case = configs.turbulence_case(24, alloc_fields=True)
    W, WA = configs.turbulence_fields(case, 5)
    steps = 4
    o = OracleSolver(case, threads=8)
    o.w[:] = W
    o.w_aux[:] = WA
    o.prepare()
    for _ in range(steps):
        o.step()
    wo, wao = o.w.copy(), o.w_aux.copy()
    o.close()
    w64, wa64 = _run(case, W, WA, "fp64", steps)
    wmx, wamx = _run(case, W, WA, "mixed", steps)
    eT64, eY64, _ = _errors(case, w64, wa64, wo, wao)
    eT, eY, eYs = _errors(case, wmx, wamx, wo, wao)
    assert eT64 < 1e-7 and eY64 < 1e-7, (eT64, eY64)
    assert eT < 1e-4 and eY < 1e-4 and eYs < 1e-12, (eT, eY, eYs)
    assert eT > 1e-12               # the FP32 paths are really taken
