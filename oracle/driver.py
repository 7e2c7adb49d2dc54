"""Python driver of the CPU oracle (test infrastructure only).

Replays the reference's ``run`` loop (src/multideal/multideal_gpu.F90:1659-1851)
on host arrays through liboracle.so.  Used by tests/ as the parity checker and
by bench.py's CPU-baseline and reference legs; the product solver never
imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "prop-streams2_b200"))

from stx.native import StxFields, load_oracle  # noqa: E402


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleSolver:
    def __init__(self, case, threads: int = 0):
        self.case = case
        self.lib = load_oracle()
        if threads:
            self.lib.ox_set_threads(threads)
        self._par, self._tab, self._grid = case.params_struct(), case.tables_struct(), case.grid_struct()
        self.ctx = self.lib.ox_ctx_create(C.byref(self._par), C.byref(self._tab), C.byref(self._grid))
        nv, ns = case.nv, case.ns
        self.w = np.ascontiguousarray(case.w.copy())
        self.w_aux = np.ascontiguousarray(case.w_aux.copy())
        shape_i = (nv, case.nz, case.ny, case.nx)
        self.fl = np.zeros(shape_i)
        self.fln = np.zeros(shape_i)
        self.fl_sav = np.zeros(shape_i)
        self.fhat = np.zeros_like(self.w)
        self.fields = StxFields(_ptr(self.w), _ptr(self.w_aux), _ptr(self.fl), _ptr(self.fln),
                                _ptr(self.fl_sav), None)
        self.time = 0.0
        self.dt = 0.0
        self.icyc = 0

    def close(self):
        if self.ctx:
            self.lib.ox_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # thin wrappers with the reference's names
    def update_ghost(self, do_swap=1):
        self.lib.ox_update_ghost_aux(self.ctx, _ptr(self.w), _ptr(self.w_aux), do_swap)

    def compute_aux(self, central=1, ghost=1):
        self.lib.ox_compute_aux(self.ctx, _ptr(self.w), _ptr(self.w_aux), central, ghost)

    def aux_slot(self, j):
        return self.w_aux[j].ctypes.data_as(C.c_void_p)

    def compute_dt(self):
        cfl = self.case.cfl
        if cfl < 0:
            self.dt = -cfl
        else:
            out = (C.c_double * 9)()
            self.lib.ox_compute_dt(self.ctx, _ptr(self.w_aux), None, out)
            self.dt = cfl / max(out)
        return self.dt

    def prepare(self):
        """Start of ``run`` (multideal_gpu.F90:1687-1727)."""
        c = self.case
        self.update_ghost(1)
        self.compute_aux(1, 1)
        self.lib.ox_bcextr_var(self.ctx, self.aux_slot(c.J("DIV")))
        self.lib.ox_bcswap(self.ctx, self.aux_slot(c.J("DIV")), 1)
        self.lib.ox_bcswap(self.ctx, self.aux_slot(c.J("DUC")), 1)
        self.fl[:] = 0.0
        self.compute_dt()

    def step(self):
        """One iteration of the ``integration`` loop (:1745-1806) without output."""
        self.icyc += 1
        if self.icyc % self.case.iter_dt_recompute == 0:
            self.compute_aux(1, 0)
            self.compute_dt()
        self.lib.ox_advance_solution(self.ctx, C.byref(self.fields), _ptr(self.fhat), self.dt, self.time)
        self.compute_aux(1, 0)
        self.time = self.time + self.dt

    def rk_sync(self, dt, simpler=0):
        self.lib.ox_rk_sync(self.ctx, C.byref(self.fields), _ptr(self.fhat), dt, simpler)

    def status(self, reset=True):
        return self.lib.ox_status(self.ctx, 1 if reset else 0)
