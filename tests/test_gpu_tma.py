"""The staged sweeps' tensor-copy staging (cp.async.bulk.tensor into shared
memory, completed on an mbarrier) against the plain staging loads, in x, y and
z: the same staged values, so the same fluxes and cell updates bit for bit.
STX_TMA=0 (read once per process) selects the plain loads, so each arm runs in
its own process.  Cases: a developed turbulence field (hybrid central / listed
WENO faces), an all-WENO field on a grid whose sizes are not multiples of the
tiles, and sweeps starting at cell 2 (characteristic boundaries), whose staged
x rows start at an odd x and land one cell into the row."""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import helpers as H  # noqa: F401

pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

_ARM = r'''
import sys, ctypes as C
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import helpers as H
from stx import configs
from stx.solver import Solver
case_kind, out = sys.argv[2], sys.argv[3]
if case_kind == "turb":
    case = configs.turbulence_case(32, alloc_fields=True)
    W, WA = configs.turbulence_fields(case, 5)
    s = Solver(case, w=torch.from_numpy(W).cuda(), w_aux=torch.from_numpy(WA).cuda())
    nmin = 1
elif case_kind == "weno":
    case = H.synthetic_case(n=(150, 37, 21), seed=3, sensor_threshold=-1.0)
    s = Solver(case)
    nmin = 1
else:
    case = H.synthetic_case(n=(150, 30, 20), seed=3, bc=(2, 2, 2, 2, 2, 2), bc_nr=(1, 1, 1, 1, 1, 1),
                            sensor_threshold=0.02, sensor_type=0)
    s = Solver(case)
    nmin = 2
s.prepare()
for _ in range(2 if case_kind == "turb" else 0):
    s.step()
s.compute_aux(1, 1)
stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
res = []
for name, n in (("x", case.nx), ("y", case.ny), ("z", case.nz)):
    for prec in (0, 1):
        s.lib.stx_set_precision(s.ctx, prec)
        fl = torch.zeros_like(s.fl)
        rc = getattr(s.lib, "stx_euler_" + name)(s.ctx, stream, C.c_void_p(s.w_aux.data_ptr()),
                                                C.c_void_p(fl.data_ptr()), nmin, n - (nmin - 1), 1)
        assert rc == 0, rc
        res.append(fl.cpu().numpy())
torch.cuda.synchronize()
assert s.status(reset=False) & 0x10 == 0          # no tensor-copy wait timed out
np.save(out, np.stack(res))
'''


@pytest.mark.parametrize("kind", ["turb", "weno", "offset"])
def test_tensor_copy_staging_equals_plain_staging(kind, tmp_path):
    here = os.path.dirname(os.path.abspath(__file__))
    outs = {}
    for arm, env in (("tma", {}), ("plain", {"STX_TMA": "0"})):
        out = str(tmp_path / f"{arm}.npy")
        r = subprocess.run([sys.executable, "-c", _ARM, here, kind, out], env=dict(os.environ, **env), cwd=here,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        outs[arm] = np.load(out)
    assert np.abs(outs["tma"]).max() > 0
    assert np.array_equal(outs["tma"], outs["plain"])
