"""The convective / viscous / transport half of the step pinned to the reference
itself: the laminar premixed flame of examples/laminar_premix_flame, run on the
GPU from the reference's own input (its multideal.ini and premix.dat), against
the reference's own FP64 run log (data.dat:32-131: rho, T, p minimum and
maximum over the domain every 1000 steps, to t = 1 ms).

The oracle check (first test) holds the GPU to the CPU restatement on the same
inputs.  The log check (second test) compares with the reference's output,
which the GPU can only match up to the transport tables: the reference built
its species viscosity, conductivity and binary-diffusion tables with Cantera
3.0.0, absent here, and this project builds them from kinetic theory (its
mixture viscosity at the inflow state is 0.7 % off the log's mu0).  Thermo and
kinetics are reproduced exactly from the mechanism file.
"""
import json
import os

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from driver import OracleSolver  # noqa: E402
from stx import configs  # noqa: E402
from stx.solver import Solver  # noqa: E402

COLS = ["rhomin", "rhomax", "tmin", "tmax", "pmin", "pmax"]


def minmax(case, w_aux):
    """compute_rho_t_p_minmax_cuf (kernels_gpu.F90:6038-6073) over the interior."""
    out = []
    for j in (case.J("R"), case.J("T"), case.J("P")):
        v = case.interior(w_aux[j])
        out += [float(v.min()), float(v.max())]
    return out


def test_flame_from_premix_matches_oracle():
    """200 steps of the reference's flame (all 2000 cells, WENO5-Z everywhere,
    KEEP(2) central part, viscous and diffusive fluxes, "simpler" splitting with
    ROK4, inflow and extrapolation boundaries) on the GPU and in the oracle."""
    case = configs.premix_flame_case()
    g = Solver(case)
    o = OracleSolver(case, threads=os.cpu_count() or 8)
    g.prepare()
    o.prepare()
    assert np.array_equal(g.host_w(), o.w)
    for _ in range(200):
        g.step()
        o.step()
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    for m in range(case.nv):
        H.assert_close(wg[m], wo[m], 1e-8, f"flame w[{m}]",
                       floor=1e-8 * np.abs(wo[:case.ns]).max() if m < case.ns else None)
    g.close()
    o.close()


def run_rows(case, nrows, graph_steps=100):
    s = Solver(case)
    s.prepare()
    graph = s.capture(graph_steps)
    rows = []
    for _ in range(nrows):
        for _ in range(1000 // graph_steps):
            s.replay(graph)
        torch.cuda.synchronize()
        rows.append(minmax(case, s.w_aux))
    s.close()
    return np.array(rows)


# Per-column bounds on the relative gap to the reference's log over all 100 rows,
# about 1.5x the gaps measured on a B200 (the GPU result is deterministic):
# rhomin 5.0e-5, rhomax 4.0e-4, tmin 1.8e-5, tmax 1.2e-5, pmin 6.2e-5, pmax 6.3e-5.
LOG_BOUNDS = {"rhomin": 7.5e-5, "rhomax": 6e-4, "tmin": 2.7e-5, "tmax": 1.8e-5, "pmin": 9.5e-5, "pmax": 9.5e-5}


def test_flame_from_premix_follows_the_reference_run_log():
    """All 100 progress rows of the reference's run (every 1000 steps to 1 ms).

    Measured on a B200, the gaps grow slowly and steadily over the run, worst
    at 1 ms for every column but rho_max: T_max 1.2e-5, T_min 1.8e-5, p
    6.3e-5, rho_min 5.0e-5, rho_max 4.0e-4 (row 83).  They come from the
    transport tables (Cantera's in the reference, kinetic theory here).  The
    pin resolves a few percent of transport: with the mixture conductivity
    scaled by 1.05 every gap grows about 3x (rho_max 1.2e-3), and with the
    binary diffusion coefficients scaled by 1.05, rho_min's gap grows to 2.6e-3
    and T_max's to 1.7e-3.  Scaling the species viscosities to the log's mu0
    (+0.75 %) changes no gap by more than 0.2 % of itself, so viscosity
    explains none of it."""
    gold = H.golden("flame_progress.json")
    ref = np.array([r[5:11] for r in gold["rows"]])
    case = configs.premix_flame_case()
    got = run_rows(case, len(ref))
    rel = np.abs(got - ref) / np.abs(ref)
    worst = {c: float(rel[:, i].max()) for i, c in enumerate(COLS)}
    print("FLAME_PIN", json.dumps(worst))
    assert np.all(np.isfinite(got))
    for c, bound in LOG_BOUNDS.items():
        assert worst[c] < bound, (c, worst)
