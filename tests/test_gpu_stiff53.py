"""The 53-species / 325-reaction synthetic stiff mechanism (stx.mech.synthetic_mechanism):
the full-Jacobian Rosenbrock step of the GPU (k_rosenbrock<53>, per-cell dense
57 x 57 Jacobian and LU) against the oracle on the same cells.

The mechanism's forward rates reach 1e22 cm^3/mol/s, so one flow step of 1e-10 s
takes the Rosenbrock integrator thousands of sub-steps from the random
(Dirichlet) initial composition; the step-size controller (relative tolerance
ros_eps = 1e-8) and the central-difference Jacobian amplify last-bit
differences, so the bar is 1e-6 relative on the state (the integrator's own
tolerance is 1e-8 per sub-step)."""
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


def test_stiff53_full_jacobian_step_matches_oracle():
    _, tb = configs.stiff_mechanism_tables(0)
    make = lambda: configs.stiff_case(1, seed=3, tables=tb, dt=1e-10, rosenbrock_version=1)
    case = make()
    assert case.ns == 53 and case.nv == 57
    o = OracleSolver(case, threads=1)
    o.prepare()
    o.step()
    g = Solver(make())
    g.prepare()
    g.step()
    torch.cuda.synchronize()
    assert o.status() & ~0x1 == 0 and g.status() & ~0x1 == 0
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    assert np.isfinite(wg).all()
    scale = np.abs(wo).reshape(case.nv, -1).max(axis=1)[:, None, None, None]
    zero = scale.ravel() == 0.0                       # the momenta of the gas at rest stay exactly zero
    assert np.array_equal(wg[zero], wo[zero])
    d = np.abs(wg - wo)[~zero] / np.maximum(np.abs(wo), 1e-6 * scale)[~zero]
    assert d.max() < 1e-6, d.max()
    Tg = case.interior(g.host_w_aux()[case.J("T")])
    To = case.interior(o.w_aux[case.J("T")])
    assert np.max(np.abs(Tg - To) / To) < 1e-6
    o.close()
    g.close()
