"""Device-side equation object: the B200 drop-in for the reference's
``equation_multideal_gpu_object`` (src/multideal/multideal_gpu.F90:164-211).

Fields live in HBM as torch tensors in the reference's SoA layout; every
kernel runs from ``libstx.so`` through its C ABI on the current torch stream.
There is no CPU path: if the CUDA library is missing, construction fails.
Method names follow the reference (``update_ghost``, ``compute_aux``,
``compute_dt``, ``rk_sync``, ``advance_solution``, ``run``).
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Optional, Sequence

import numpy as np
import torch

from .native import StxFields, StxTuning, check, load_stx


def _p(t: Optional[torch.Tensor]):
    return None if t is None else C.c_void_p(t.data_ptr())


class Solver:
    def __init__(self, case, device: str = "cuda", w: Optional[torch.Tensor] = None,
                 w_aux: Optional[torch.Tensor] = None, aux_slots: Optional[Sequence[int]] = None,
                 tables_from: Optional["Solver"] = None, stream_ordered: bool = False):
        """case: a Case; w, w_aux: device fields to use in place of the case's host
        fields.  aux_slots: upload only these (0-based) slots of case.w_aux, the
        others starting at zero -- for a fresh case only the temperature slot
        (the Newton iteration's first guess) holds data before eval_aux.
        tables_from: a live solver of the same mechanism whose device tables
        this one uses (stx_ctx_create_like); it must outlive this one.
        stream_ordered (with tables_from): the context's uploads are enqueued on
        the current stream instead of waited for (stx_ctx_create_like_on), so
        creating the solver waits for no other work on the device; use it on
        that stream."""
        if not torch.cuda.is_available():
            raise RuntimeError("the stx solver needs a CUDA device (there is no CPU fallback)")
        self.lib = load_stx()
        self.case = case
        dev = torch.device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        torch.cuda.set_device(self.device)
        self._par, self._tab, self._grid = case.params_struct(), case.tables_struct(), case.grid_struct()
        ctx = C.c_void_p()
        if tables_from is not None:
            if tables_from.case.ns != case.ns or not tables_from.ctx:
                raise ValueError("tables_from must be a live solver of the same mechanism")
            if stream_ordered:
                check(self.lib.stx_ctx_create_like_on(tables_from.ctx, C.byref(self._par), C.byref(self._grid),
                                                      self.stream, C.byref(ctx)), "stx_ctx_create_like_on")
            else:
                check(self.lib.stx_ctx_create_like(tables_from.ctx, C.byref(self._par), C.byref(self._grid),
                                                   C.byref(ctx)), "stx_ctx_create_like")
        else:
            check(self.lib.stx_ctx_create(C.byref(self._par), C.byref(self._tab), C.byref(self._grid), C.byref(ctx)),
                  "stx_ctx_create")
        self.ctx = ctx
        nv = case.nv
        # host fields go up through pinned staging, asynchronously on the current
        # stream (the kernels that follow on it see them)
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().to(self.device, non_blocking=True)
        if w is None:
            w = up(case.w)
        if w_aux is None:
            if aux_slots is None:
                w_aux = up(case.w_aux)
            else:      # only these slots hold data; the others start at zero
                w_aux = torch.zeros(case.w_aux.shape, dtype=torch.float64, device=self.device)
                for j in aux_slots:
                    w_aux[j].copy_(up(case.w_aux[j]), non_blocking=True)
        self.w = w.contiguous()
        self.w_aux = w_aux.contiguous()
        assert self.w.shape == (nv, case.nzg, case.nyg, case.nxg) and self.w.dtype == torch.float64
        assert self.w_aux.shape == (case.nv_aux, case.nzg, case.nyg, case.nxg)
        shp = (nv, case.nz, case.ny, case.nx)
        self.fl = torch.zeros(shp, dtype=torch.float64, device=self.device)
        self.fln = torch.zeros(shp, dtype=torch.float64, device=self.device)
        self.fl_sav = torch.zeros(shp, dtype=torch.float64, device=self.device)
        self.fields = StxFields(self.w.data_ptr(), self.w_aux.data_ptr(), self.fl.data_ptr(), self.fln.data_ptr(),
                                self.fl_sav.data_ptr(), None)
        self.time = 0.0
        self.dt = 0.0
        self.icyc = 0

    # ------------------------------------------------------------------ plumbing
    @property
    def stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def close(self):
        for g in getattr(self, "_graphs", []):
            self.lib.stx_graph_destroy(g)
        self._graphs = []
        if getattr(self, "ctx", None):
            self.lib.stx_ctx_destroy(self.ctx)
            self.ctx = None

    # ------------------------------------------------------------------ captured steps
    def capture(self, nsteps: int):
        """Capture nsteps iterations of the integration loop into one CUDA graph
        (iter_dt_recompute = 1).  Fixed dt (cfl < 0): the step size is known; a
        CFL-driven run (cfl > 0): every captured step forms its dt from the CFL
        maxima on the device.  Replaying it with ``replay`` gives the same result
        as nsteps calls of ``step``."""
        if self.case.iter_dt_recompute != 1:
            raise ValueError("captured steps need iter_dt_recompute = 1")
        g = C.c_void_p()
        if self.case.cfl < 0:
            self.dt = -self.case.cfl
            check(self.lib.stx_graph_create(self.ctx, C.byref(self.fields), self.dt, nsteps, C.byref(g)),
                  "stx_graph_create")
        else:
            check(self.lib.stx_graph_create_cfl(self.ctx, C.byref(self.fields), self.case.cfl, nsteps, C.byref(g)),
                  "stx_graph_create_cfl")
        if not hasattr(self, "_graphs"):
            self._graphs = []
        self._graphs.append(g)
        return g, nsteps

    def replay(self, graph):
        """Launch a captured graph.  A CFL-driven graph's time and last dt are
        read back (one synchronisation per replay)."""
        g, n = graph
        check(self.lib.stx_graph_launch(g, self.stream, self.time), "stx_graph_launch")
        self.icyc += n
        if self.case.cfl < 0:
            for _ in range(n):
                self.time = self.time + self.dt
        else:
            t, dt = C.c_double(), C.c_double()
            check(self.lib.stx_graph_state(g, self.stream, C.byref(t), C.byref(dt)), "stx_graph_state")
            self.time, self.dt = t.value, dt.value

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, form: str):
        """"fp64" (the reference method, default) or "mixed" (FP32 face fluxes and
        transport properties, FP64 residual, Newton and chemistry)."""
        mode = {"fp64": 0, "mixed": 1}[form]
        check(self.lib.stx_set_precision(self.ctx, mode), "stx_set_precision")
        self.precision = form

    # ------------------------------------------------------------------ tuning
    def tuning(self) -> dict:
        """The context's launch choices (stx_get_tuning)."""
        t = StxTuning()
        check(self.lib.stx_get_tuning(self.ctx, C.byref(t)), "stx_get_tuning")
        return _tuning_dict(t)

    def set_tuning(self, tune: dict):
        t = StxTuning()
        t.sweep_kind[:] = tune["sweep_kind"]
        t.weno_list[:] = tune["weno_list"]
        t.chem_ctas_per_sm = tune["chem_ctas_per_sm"]
        t.batch_ctas_max = tune.get("batch_ctas_max", 0)
        check(self.lib.stx_set_tuning(self.ctx, C.byref(t)), "stx_set_tuning")

    def tuning_key(self) -> str:
        c = self.case
        return (f"{torch.cuda.get_device_name(self.device)}|ns={c.ns}|{c.nx}x{c.ny}x{c.nz}|ep={c.ep_order}|"
                f"weno={c.weno_scheme}|chem={c.enable_chemistry}/{c.rosenbrock_version}|"
                f"prec={getattr(self, 'precision', 'fp64')}")

    def autotune(self, dt_chem: Optional[float] = None, cache: Optional[str] = None) -> dict:
        """Choose the launch shapes by timing them (stx_autotune) on the current
        fields, which must be prepared (``prepare``); they are not modified.
        dt_chem: the chemistry window to time (default: half of the current dt,
        the Strang half step).  cache: a JSON file of earlier choices keyed by
        device, species count, grid, scheme and precision; a hit applies the
        stored choice without timing, a miss times and adds it."""
        key = self.tuning_key()
        if cache and os.path.exists(cache):
            with open(cache) as fh:
                known = json.load(fh)
            if key in known:
                self.set_tuning(known[key])
                return dict(known[key], cached=True)
        t = StxTuning()
        dtc = 0.5 * self.dt if dt_chem is None else dt_chem
        check(self.lib.stx_autotune(self.ctx, self.stream, C.byref(self.fields), dtc, C.byref(t)), "stx_autotune")
        out = _tuning_dict(t)
        if cache:
            known = {}
            if os.path.exists(cache):
                with open(cache) as fh:
                    known = json.load(fh)
            known[key] = out
            with open(cache, "w") as fh:
                json.dump(known, fh, indent=1, sort_keys=True)
        return dict(out, cached=False)

    def aux_slot(self, j: int) -> C.c_void_p:
        return C.c_void_p(self.w_aux[j].data_ptr())

    def status(self, reset: bool = True) -> int:
        b = C.c_uint32()
        check(self.lib.stx_status(self.ctx, self.stream, C.byref(b), 1 if reset else 0), "stx_status")
        return b.value

    # ------------------------------------------------------------------ reference-named calls
    def update_ghost(self, do_swap: int = 1):
        check(self.lib.stx_update_ghost_aux(self.ctx, self.stream, _p(self.w), _p(self.w_aux), do_swap),
              "update_ghost")

    def compute_aux(self, central: int = 1, ghost: int = 1):
        check(self.lib.stx_compute_aux(self.ctx, self.stream, _p(self.w), _p(self.w_aux), central, ghost), "compute_aux")

    def compute_dt(self) -> float:
        cfl = self.case.cfl
        if cfl < 0:
            self.dt = -cfl
        else:
            out = (C.c_double * 9)()
            check(self.lib.stx_compute_dt(self.ctx, self.stream, _p(self.w_aux), None, out), "compute_dt")
            self.dt = cfl / max(out)
        return self.dt

    def rk_sync(self, dt: Optional[float] = None, simpler: int = 0):
        check(self.lib.stx_rk_sync(self.ctx, self.stream, C.byref(self.fields), self.dt if dt is None else dt, simpler),
              "rk_sync")

    def advance_solution(self):
        check(self.lib.stx_advance_solution(self.ctx, self.stream, C.byref(self.fields), self.dt, self.time),
              "advance_solution")

    def prepare(self):
        """Start of ``run`` (multideal_gpu.F90:1687-1727)."""
        c = self.case
        self.update_ghost(1)
        self.compute_aux(1, 1)
        check(self.lib.stx_bcextr_var(self.ctx, self.stream, self.aux_slot(c.J("DIV"))), "bcextr_var")
        check(self.lib.stx_bcswap(self.ctx, self.stream, self.aux_slot(c.J("DIV")), 1), "bcswap_var")
        check(self.lib.stx_bcswap(self.ctx, self.stream, self.aux_slot(c.J("DUC")), 1), "bcswap_var")
        self.fl.zero_()
        self.compute_dt()

    def step(self, recompute_dt: bool = True):
        """One iteration of the reference's ``integration`` loop (:1745-1806), no output."""
        self.icyc += 1
        if recompute_dt and self.icyc % self.case.iter_dt_recompute == 0:
            self.compute_aux(1, 0)
            self.compute_dt()
        self.advance_solution()
        self.compute_aux(1, 0)
        self.time = self.time + self.dt

    def run(self, num_iter: int):
        self.prepare()
        for _ in range(num_iter):
            self.step()

    # ------------------------------------------------------------------ host views
    def host_w(self) -> np.ndarray:
        return self.w.cpu().numpy()

    def host_w_aux(self) -> np.ndarray:
        return self.w_aux.cpu().numpy()


def _tuning_dict(t: StxTuning) -> dict:
    return {"sweep_kind": list(t.sweep_kind), "weno_list": list(t.weno_list), "chem_ctas_per_sm": t.chem_ctas_per_sm,
            "chem_ctas_max": t.chem_ctas_max, "batch_ctas_max": t.batch_ctas_max,
            "sweep_ms": [round(x, 4) for x in t.sweep_ms],
            "chem_ms": round(t.chem_ms, 4)}
