"""The allocation-free ROK4 entry point (stx_rosenbrock_krylov_noalloc).

It exists for callers that cannot call cudaMalloc -- device memory owned by
another runtime or a fixed pool, or a path that must not allocate while work
is in flight -- so it takes the caller's own device tables and fields, needs
no context, and keeps its only scratch (the work-stealing cell counter) in a
file-scope device array.  Its kernel's per-thread working set lives in local
memory, which the driver grows by a device allocation when a launch needs more
than cudaLimitStackSize; the entry point refuses such a launch
(STX_E_LOCAL_MEM), so the caller sets that limit once at initialisation.

Here it must give the same result as the context path (stx_rosenbrock_krylov)
on two consecutive calls, for both splittings; leave the free device memory
unchanged on its first launch in a fresh process; refuse a stack limit below
its frame; and refuse a problem larger than its scratch allows.

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from stx.native import StxGrid, StxTables, load_stx  # noqa: E402
from stx.solver import Solver  # noqa: E402

FN = "stx_rosenbrock_krylov_noalloc"
E_LOCAL_MEM = -6
# per-thread stack limit a caller sets once for up to 14 species (include/stx.h)
STACK_BYTES = 4608


def set_stack_limit(nbytes):
    """cudaDeviceSetLimit(cudaLimitStackSize) on the current device's primary
    context (the one torch and libstx use); returns the limit now in force."""
    from cuda.bindings import runtime as rt
    err, = rt.cudaDeviceSetLimit(rt.cudaLimit.cudaLimitStackSize, nbytes)
    assert err == rt.cudaError_t.cudaSuccess, err
    err, val = rt.cudaDeviceGetLimit(rt.cudaLimit.cudaLimitStackSize)
    assert err == rt.cudaError_t.cudaSuccess, err
    return val


def _bind(lib):
    fn = getattr(lib, FN)
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p]
    return fn


class DeviceTables:
    """The tables of a case uploaded to the device by the caller, in the
    reference's Fortran layouts (as a Fortran host would hold them)."""

    def __init__(self, case, dev):
        host = case.tables_struct()
        self.keep = []
        self.t = StxTables()
        for name, ctype in StxTables._fields_:
            val = getattr(host, name)
            if isinstance(val, int) or isinstance(val, float):
                setattr(self.t, name, val)
        n = {"mw": case.ns, "mwinv": case.ns, "rgas": case.ns, "trange": case.tb.trange.size,
             "cp_coeff": case.tb.cp_coeff.size, "cv_coeff": case.tb.cv_coeff.size,
             "reac_ty": case.tb.nr, "is_rev": case.tb.nr, "arr_a": 2 * case.tb.nr, "arr_b": 2 * case.tb.nr,
             "arr_ea": 2 * case.tb.nr, "falloff": 5 * case.tb.nr, "tb_eff": case.tb.nr * case.ns,
             "r_coeffs": case.tb.nr * case.ns, "p_coeffs": case.tb.nr * case.ns,
             "kc_tab": (case.tb.num_t_tab + 1) * case.tb.nr}
        for name, count in n.items():
            src = getattr(host, name)
            is_int = name in ("reac_ty", "is_rev")
            arr = np.ctypeslib.as_array(src, shape=(count,)).copy()
            t = torch.from_numpy(arr).to(dev)
            self.keep.append(t)
            setattr(self.t, name, C.cast(C.c_void_p(t.data_ptr()),
                                         C.POINTER(C.c_int32) if is_int else C.POINTER(C.c_double)))


def _run_pair(case, simpler):
    """Two chained calls of the context path and of the allocation-free entry
    point from the same state; returns the fields after each call."""
    dev = torch.device("cuda", torch.cuda.current_device())
    set_stack_limit(STACK_BYTES)
    ref = Solver(case)                      # context path (allocates at creation)
    ref.update_ghost(1)
    ref.compute_aux(1, 1)
    w0 = ref.w.clone()
    wa = ref.w_aux.clone()
    fl_sav = None
    if simpler:
        # a residual for the "simpler" splitting's fl_sav, the same for both paths
        rng = np.random.default_rng(7)
        scale = np.abs(ref.w.cpu().numpy()).max(axis=(1, 2, 3)) * 1e3
        fs = rng.standard_normal(ref.fl_sav.shape) * scale[:, None, None, None]
        fl_sav = torch.from_numpy(fs).to(dev)
    fn = _bind(load_stx())
    dt_tabs = DeviceTables(case, dev)
    grid = StxGrid()
    grid.nx, grid.ny, grid.nz, grid.ng = case.nx, case.ny, case.nz, case.ng
    par = case.params_struct()
    w = w0.clone()
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    fsp = None if fl_sav is None else C.c_void_p(fl_sav.data_ptr())
    dt_chem = 2e-7
    outs = []
    for call in range(2):
        t0, t1 = call * dt_chem, (call + 1) * dt_chem
        rc = ref.lib.stx_rosenbrock_krylov(ref.ctx, ref.stream, C.c_void_p(ref.w.data_ptr()),
                                           C.c_void_p(wa.data_ptr()), fsp, dt_chem, t0, t1, simpler)
        assert rc == 0
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = fn(C.byref(par), C.byref(dt_tabs.t), C.byref(grid), stream, C.c_void_p(w.data_ptr()),
                C.c_void_p(wa.data_ptr()), fsp, dt_chem, t0, t1, simpler, C.c_void_p(status.data_ptr()))
        assert rc == 0, load_stx().stx_strerror(rc)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info(dev)[0] == free_before    # nothing allocated by the call
        outs.append((ref.w.cpu().numpy().copy(), w.cpu().numpy().copy()))
    ref.close()
    return outs, status


@pytest.mark.parametrize("simpler", [0, 1])
def test_noalloc_matches_context_path_on_two_calls(simpler):
    case = H.synthetic_case(n=(10, 8, 6), seed=21, T0=1300.0, amp_T=200.0)
    outs, status = _run_pair(case, simpler)
    for a, b in outs:
        for m in range(case.nv):
            H.assert_close(case.interior(b[m]), case.interior(a[m]), 1e-9, f"noalloc w[{m}] simpler={simpler}",
                           floor=1e-9 * np.abs(case.interior(a[:case.ns])).max() if m < case.ns else None)
    # the second call continues from the first
    assert not np.array_equal(outs[0][1], outs[1][1])


def test_noalloc_rejects_problems_beyond_its_scratch():
    case = H.synthetic_case(n=(4, 4, 4), seed=22)
    fn = _bind(load_stx())
    grid = StxGrid()
    grid.nx, grid.ny, grid.nz, grid.ng = 2048, 1024, 1025, 3            # > 2^31 cells
    par = case.params_struct()
    tabs = DeviceTables(case, torch.device("cuda", torch.cuda.current_device()))
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = fn(C.byref(par), C.byref(tabs.t), C.byref(grid), None, C.c_void_p(dummy.data_ptr()),
            C.c_void_p(dummy.data_ptr()), None, 1e-7, 0.0, 1e-7, 0, None)
    assert rc == -5
    assert b"2^31" in load_stx().stx_strerror(rc)


# Run in a fresh interpreter, so that the allocation-free entry point is the
# first libstx code to touch the device: the caller's one-time set-up, then the
# first launch, which must leave the free device memory exactly unchanged.
_FRESH = r'''
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import helpers as H
import test_zz_no_alloc as T
from stx.native import StxGrid, load_stx
dev = torch.device("cuda", 0)
torch.cuda.set_device(dev)
case = H.synthetic_case(n=(10, 8, 6), seed=23, T0=1300.0, amp_T=200.0)
# caller-owned device memory: tables, fields, status word (all before any call)
tabs = T.DeviceTables(case, dev)
w = torch.from_numpy(np.ascontiguousarray(case.w)).to(dev)
wa = torch.from_numpy(np.ascontiguousarray(case.w_aux)).to(dev)
wa[case.J("Z")] = 0.5          # the Bilger Z eval_aux gives with one element of interest
status = torch.zeros(1, dtype=torch.int32, device=dev)
grid = StxGrid(); grid.nx, grid.ny, grid.nz, grid.ng = case.nx, case.ny, case.nz, case.ng
par = case.params_struct()
fn = T._bind(load_stx())
stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
args = lambda: (C.byref(par), C.byref(tabs.t), C.byref(grid), stream, C.c_void_p(w.data_ptr()),
                C.c_void_p(wa.data_ptr()), None, 1e-7, 0.0, 1e-7, 0, C.c_void_p(status.data_ptr()))
torch.cuda.synchronize()
# 1. a stack limit below the kernel's frame: refused, nothing launched (this
#    first call does the set-up: the kernel is loaded, the scratch looked up)
T.set_stack_limit(1024)
w_before = w.clone(); torch.cuda.synchronize()
rc = fn(*args())
torch.cuda.synchronize()
assert rc == T.E_LOCAL_MEM, rc
assert torch.equal(w, w_before)
# 2. the caller's one-time initialisation
T.set_stack_limit(T.STACK_BYTES)
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info(dev)[0]
# 3. the first launch allocates nothing
rc = fn(*args())
torch.cuda.synchronize()
assert rc == 0, rc
free1 = torch.cuda.mem_get_info(dev)[0]
assert free1 == free0, (free0, free1)
assert not torch.equal(w, w_before)
print("FRESH_OK", free0 - free1)
'''


@pytest.mark.parametrize("loading", ["LAZY", "EAGER"])
def test_noalloc_first_launch_in_a_fresh_process_allocates_nothing(loading):
    env = dict(os.environ, CUDA_MODULE_LOADING=loading)
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run([sys.executable, "-c", _FRESH, here], env=env, cwd=here, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and "FRESH_OK 0" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]
