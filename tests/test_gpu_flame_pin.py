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
# about 1.3x the gaps measured on a B200: rhomin 2.6e-3, rhomax 4.7e-3,
# tmin 9.4e-4, tmax 6.9e-4, pmin 3.3e-3, pmax 3.2e-3 (the worst rows are the
# first 10-20, 1e4-2e4 steps in; at 1 ms the gaps are rhomin 1.0e-4,
# rhomax 3.5e-3, tmin 3.3e-5, tmax 2.4e-6, pmin 1.2e-4, pmax 3.4e-5).
LOG_BOUNDS = {"rhomin": 3.5e-3, "rhomax": 6e-3, "tmin": 1.3e-3, "tmax": 1e-3, "pmin": 4.5e-3, "pmax": 4.5e-3}


def test_flame_from_premix_follows_the_reference_run_log():
    """All 100 progress rows of the reference's run (every 1000 steps to 1 ms).

    The gap is a start-up transient, not drift: premix.dat is a steady flame for
    the reference's (Cantera) transport, so the reference's pressure stays within
    20 Pa of 101320 Pa, while with this project's kinetic-theory tables the flame
    first readjusts and sends an acoustic transient through the domain (the
    pressure dips by up to 330 Pa near 1e4 steps, the inlet temperature follows
    it isentropically) that has decayed by 1 ms, where T_max agrees to 2.4e-6.
    rho_max, set by the composition of the cold preheat zone (species
    diffusion), keeps a 3.5e-3 gap.  Scaling the species viscosities to the
    log's mu0 (+0.75 %) changes every column's worst gap by at most 0.1 % of
    itself, so viscosity explains none of it."""
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
    # the transient decays: the last row is far closer than the worst one for T and p
    last = rel[-1]
    assert last[COLS.index("tmax")] < 1e-5 and last[COLS.index("pmin")] < 5e-4 and last[COLS.index("pmax")] < 5e-4
