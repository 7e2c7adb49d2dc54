"""The autotuner and the launch choices it picks among (stx_autotune,
stx_get_tuning / stx_set_tuning).

* The autotuner leaves the caller's fields and status word untouched and keeps
  a valid choice; a cache file replays it without timing.
* Listed WENO faces (k_weno_list) and WENO computed in line give the same
  fields bit for bit; so do different persistent CTA counts of the chemistry.
* The staged-tile and one-face-per-thread sweeps agree to rounding (their
  FP64 expressions contract to FMAs differently)."""
import numpy as np
import pytest
import torch

import helpers as H  # noqa: F401  (puts the package on sys.path)

pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from stx import configs  # noqa: E402
from stx.native import check  # noqa: E402
from stx.solver import Solver  # noqa: E402

BASE = {"sweep_kind": [0, 0, 0], "weno_list": [1, 1, 1], "chem_ctas_per_sm": 0}


def _turb(n=24, seed=5, **over):
    case = configs.turbulence_case(n, alloc_fields=True, **over)
    W, WA = configs.turbulence_fields(case, seed)
    s = Solver(case, w=torch.from_numpy(W).cuda(), w_aux=torch.from_numpy(WA).cuda())
    s.prepare()
    return s


def _steps(make, tune, nsteps):
    s = make()
    s.set_tuning(tune)
    for _ in range(nsteps):
        s.step()
    torch.cuda.synchronize()
    w, wa = s.host_w(), s.host_w_aux()
    s.close()
    return w, wa


def test_autotune_leaves_fields_and_keeps_a_valid_choice(tmp_path):
    s = _turb()
    torch.cuda.synchronize()
    w0, wa0, st0 = s.w.clone(), s.w_aux.clone(), s.status(reset=False)
    t = s.autotune(cache=str(tmp_path / "tune.json"))
    torch.cuda.synchronize()
    assert torch.equal(s.w, w0) and torch.equal(s.w_aux, wa0)
    assert s.status(reset=False) == st0
    assert not t["cached"]
    assert all(k in (0, 1) for k in t["sweep_kind"] + t["weno_list"])
    assert -1 <= t["chem_ctas_per_sm"] <= t["chem_ctas_max"] and t["chem_ctas_max"] >= 1
    assert all(ms > 0 for ms in t["sweep_ms"]) and t["chem_ms"] > 0
    got = s.tuning()
    assert got["sweep_kind"] == t["sweep_kind"] and got["weno_list"] == t["weno_list"]
    s.close()
    s2 = _turb()
    t2 = s2.autotune(cache=str(tmp_path / "tune.json"))
    assert t2["cached"] and t2["sweep_kind"] == t["sweep_kind"]
    assert s2.tuning()["chem_ctas_per_sm"] == t["chem_ctas_per_sm"]
    s2.close()


def test_listed_weno_and_cta_counts_are_bit_identical():
    # negative Ducros threshold: every face takes the WENO flux (the reference's examples)
    make = lambda: _turb(16, seed=3, sensor_threshold=-0.2)
    w_a, wa_a = _steps(make, BASE, 2)
    w_b, wa_b = _steps(make, dict(BASE, weno_list=[0, 0, 0]), 2)
    w_c, wa_c = _steps(make, dict(BASE, chem_ctas_per_sm=1), 2)
    # the plain launch: one thread per cell, no work stealing
    w_d, wa_d = _steps(make, dict(BASE, chem_ctas_per_sm=-1), 2)
    assert np.array_equal(w_a, w_b) and np.array_equal(wa_a, wa_b)
    assert np.array_equal(w_a, w_c) and np.array_equal(wa_a, wa_c)
    assert np.array_equal(w_a, w_d) and np.array_equal(wa_a, wa_d)


@pytest.mark.parametrize("thr", [0.1, -0.2])
def test_staged_and_per_face_sweeps_agree(thr):
    """The convective residual of each sweep direction from both kernels, on the
    same fields (after two steps, so the Ducros sensor marks faces)."""
    import ctypes as C
    s = _turb(16, seed=7, sensor_threshold=thr)
    for _ in range(2):
        s.step()
    s.compute_aux(1, 0)
    out = {}
    for name, tune in (("staged", BASE), ("face", dict(BASE, sweep_kind=[1, 1, 1], weno_list=[0, 0, 0]))):
        s.set_tuning(tune)
        fl = torch.empty_like(s.fl)
        for d, fn in enumerate((s.lib.stx_euler_x, s.lib.stx_euler_y, s.lib.stx_euler_z)):
            n = (s.case.nx, s.case.ny, s.case.nz)[d]
            check(fn(s.ctx, s.stream, C.c_void_p(s.w_aux.data_ptr()), C.c_void_p(fl.data_ptr()), 1, n,
                     1 if d == 0 else 0), "euler sweep")
        torch.cuda.synchronize()
        out[name] = fl.cpu().numpy()
    s.close()
    a, b = out["staged"], out["face"]
    for m in range(a.shape[0]):
        scale = np.max(np.abs(b[m])) + 1e-300
        assert np.max(np.abs(a[m] - b[m])) / scale < 1e-12, m
