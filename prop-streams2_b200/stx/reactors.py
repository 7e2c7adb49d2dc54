"""Batched adiabatic constant-pressure 0-D reactors on the GPU.

The reference integrates one 0-D reactor per run (examples/batch_reactor:
flow_init 8, a single constant-volume cell pushed through the whole solver,
multideal.F90:5305-5381).  Here many reactors of different initial states run
in one persistent launch of stx_batch0d_integrate: every thread integrates
one reactor with the reference's ROK4 scheme (kernels_gpu.F90:10360-11205),
claiming the next reactor when it is done, so reactors that ignite late do
not hold up the others.  The formulation is constant pressure (state Y_k,
enthalpy and pressure fixed; T from h as get_mixture_temperature_from_h_roe_dev,
kernels_gpu.F90:6810-6900).  The ignition time is the first accepted time at
which T > ign_factor * T0 (the T > 1.05 T0 test of
examples/syngas_mech_eval/mech_comp.py); integration stops at
min(t_max, end_factor * t_ign).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Union

import numpy as np
import torch

from . import case as CS
from . import configs
from . import mech as M
from .native import check, load_stx


class BatchReactors:
    """A context holding one mechanism's tables for batched reactor solves."""

    def __init__(self, mechanism: Union[str, M.Mechanism] = "h2air_9sp", device: str = "cuda",
                 tables: Optional[M.Tables] = None, tol_iter_nr: float = 1e-12):
        if not torch.cuda.is_available():
            raise RuntimeError("BatchReactors needs a CUDA device (there is no CPU fallback)")
        self.lib = load_stx()
        mech = configs.mechanism(mechanism) if isinstance(mechanism, str) else mechanism
        self.mech = mech
        if tables is None:
            tables = M.build_tables(mech, 101325.0, 200.0, 5500.0, 1.0)
        Y = np.full(mech.ns, 1.0 / mech.ns)
        cfg = CS.default_ini(1, 1, 1, L=(1e-3, 1e-3, 1e-3), Y=Y, ns=mech.ns, chemistry=2, rosenbrock_version=2)
        self.case = CS.Case(cfg, tables, alloc_fields=False)
        self.case.tol_iter_nr = tol_iter_nr
        dev = torch.device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        torch.cuda.set_device(dev)
        self._par, self._tab, self._grid = self.case.params_struct(), self.case.tables_struct(), self.case.grid_struct()
        ctx = C.c_void_p()
        check(self.lib.stx_ctx_create(C.byref(self._par), C.byref(self._tab), C.byref(self._grid), C.byref(ctx)),
              "stx_ctx_create")
        self.ctx = ctx

    @property
    def ns(self) -> int:
        return self.mech.ns

    def stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def integrate(self, T0, p0, Y0, t_max: float, dttry: float = 1e-8, ign_factor: float = 1.05,
                  end_factor: float = 2.0, max_steps: int = 100000, sync: bool = True,
                  order: str = "given") -> dict:
        """Integrate n reactors.  T0, p0: (n,); Y0: (ns, n) mass fractions (reactor
        index fastest).  Tensors already on the device are used in place; numpy
        arrays are copied to the device.  Returns device tensors Y (ns, n), T,
        t_ign (-1 where no ignition), t_end, nsteps.

        order="coldest_first" hands the reactors to the work-stealing schedule in
        order of rising T0 (the cold ones have the longest ignition delays and
        the most steps), so the longest integrations start first and the tail of
        the launch shortens.  A reactor's result does not depend on the order."""
        f64 = dict(dtype=torch.float64, device=self.device)
        T0 = torch.as_tensor(T0, **f64).contiguous()
        p0 = torch.as_tensor(p0, **f64).contiguous()
        Y0 = torch.as_tensor(Y0, **f64).contiguous()
        n = T0.numel()
        if p0.numel() != n or Y0.shape != (self.ns, n):
            raise ValueError(f"expected T0, p0 of shape ({n},) and Y0 of shape ({self.ns}, {n})")
        if order not in ("given", "coldest_first"):
            raise ValueError(f"unknown order {order!r}")
        if order == "coldest_first" and n > 1:
            perm = torch.argsort(T0)
            out = self.integrate(T0[perm], p0[perm], Y0[:, perm].contiguous(), t_max, dttry, ign_factor,
                                 end_factor, max_steps, sync=False)
            inv = torch.empty_like(perm)
            inv[perm] = torch.arange(n, device=self.device)
            res = {k: (v[:, inv] if v.dim() == 2 else v[inv]) for k, v in out.items()}
            if sync:
                torch.cuda.current_stream(self.device).synchronize()
            return res
        out = dict(Y=torch.empty_like(Y0), T=torch.empty_like(T0), t_ign=torch.empty_like(T0),
                   t_end=torch.empty_like(T0), nsteps=torch.empty(n, dtype=torch.int32, device=self.device))
        vp = lambda t: C.c_void_p(t.data_ptr())
        check(self.lib.stx_batch0d_integrate(self.ctx, self.stream(), n, vp(T0), vp(p0), vp(Y0), t_max, dttry,
                                             ign_factor, end_factor, max_steps, vp(out["Y"]), vp(out["T"]),
                                             vp(out["t_ign"]), vp(out["t_end"]), vp(out["nsteps"])),
              "stx_batch0d_integrate")
        if sync:
            torch.cuda.current_stream(self.device).synchronize()
        return out

    def launch(self, T0: torch.Tensor, p0: torch.Tensor, Y0: torch.Tensor, out: dict, t_max: float,
               dttry: float = 1e-8, ign_factor: float = 1.05, end_factor: float = 2.0, max_steps: int = 100000):
        """Launch n reactors on the current stream with caller-owned buffers and
        return at once.  Every tensor is either on the device or in pinned host
        memory (read and written by the kernel in place, no copies): T0, p0 (n,),
        Y0 (ns, n) float64 contiguous; out holds Y, T, t_ign, t_end (float64) and
        nsteps (int32) of the same shapes.  The kernel writes a reactor's nsteps
        after its other outputs, behind a system-scope fence, so with nsteps in
        pinned host memory preset to -1 the caller can collect each reactor as
        soon as its nsteps turns non-negative, before the launch ends."""
        n = T0.numel()
        ts = [T0, p0, Y0] + [out[k] for k in ("Y", "T", "t_ign", "t_end", "nsteps")]
        for t in ts:
            if not t.is_contiguous() or not (t.is_cuda or t.is_pinned()):
                raise ValueError("launch needs contiguous device or pinned host tensors")
        if p0.numel() != n or tuple(Y0.shape) != (self.ns, n) or tuple(out["Y"].shape) != (self.ns, n):
            raise ValueError(f"expected T0, p0 of shape ({n},) and Y0, Y of shape ({self.ns}, {n})")
        if any(out[k].numel() != n for k in ("T", "t_ign", "t_end", "nsteps")) or out["nsteps"].dtype != torch.int32:
            raise ValueError("out: T, t_ign, t_end float64 and nsteps int32 of n entries")
        vp = lambda t: C.c_void_p(t.data_ptr())
        check(self.lib.stx_batch0d_integrate(self.ctx, self.stream(), n, vp(T0), vp(p0), vp(Y0), t_max, dttry,
                                             ign_factor, end_factor, max_steps, vp(out["Y"]), vp(out["T"]),
                                             vp(out["t_ign"]), vp(out["t_end"]), vp(out["nsteps"])),
              "stx_batch0d_integrate")

    def set_form(self, form: str):
        """"fp64" (the reference method, default) or "split": the FP32/FP64-split
        form, with the Krylov basis and the stage vectors of ROK4 stored in FP32
        and the state, every right-hand side and the error control in FP64 (the
        context's mixed precision form)."""
        mode = {"fp64": 0, "split": 1}[form]
        check(self.lib.stx_set_precision(self.ctx, mode), "stx_set_precision")

    def set_launch_cap(self, ctas: int):
        """Cap the CTAs of this context's launches (0: none), so that several
        reactor launches running at once leave SMs for other work: the
        persistent kernels hold their CTAs until the last reactor is done."""
        from .native import StxTuning
        t = StxTuning()
        check(self.lib.stx_get_tuning(self.ctx, C.byref(t)), "stx_get_tuning")
        t.batch_ctas_max = int(ctas)
        check(self.lib.stx_set_tuning(self.ctx, C.byref(t)), "stx_set_tuning")

    def status(self, reset: bool = True) -> int:
        bits = C.c_uint32()
        check(self.lib.stx_status(self.ctx, self.stream(), C.byref(bits), int(reset)), "stx_status")
        return bits.value

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.stx_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sample_h2air(n: int, seed: int, mech: M.Mechanism, T_range=(900.0, 1500.0), p_atm=(1.0, 40.0),
                 phi_range=(0.3, 3.0)):
    """The batched-reactor workload: T0 ~ U(900, 1500) K, p ~ logU(1, 40) atm,
    phi ~ U(0.3, 3), H2/air (O2:N2 = 1:3.76), seeded.  Returns numpy T0 (n,),
    p0 (n,), Y0 (ns, n)."""
    rng = np.random.default_rng(seed)
    T0 = rng.uniform(*T_range, n)
    p0 = 101325.0 * np.exp(rng.uniform(np.log(p_atm[0]), np.log(p_atm[1]), n))
    phi = rng.uniform(*phi_range, n)
    Y0 = np.stack([configs.h2air_Y(f, mech) for f in phi], axis=1)
    return T0, p0, Y0
