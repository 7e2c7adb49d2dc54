"""Output and restart files of the reference's run, for the examples on this path.

The writers reproduce the reference's file formats, so that its own comparison
scripts (``examples/*/OUTPUT/result_comp.py``) and its restart reader take the
files of this implementation:

* ``progress.out`` lines of ``print_progress`` (src/multideal/multideal_gpu.F90:1933-1972):
  ``'(1I10,F18.10,20ES20.10)'`` icyc, step time, dt, time, residual, rho/T/p extrema;
* ``output_1d_{170,190,230}micro_s.dat`` of the reactive shock tube, ``output_LPF.dat``
  of the premixed flame and ``output_batch.dat`` of the batch reactor (``manage_output``,
  multideal_gpu.F90:2518-2564);
* the restart: ``rst1_XXXX_XXXX_XXXX.bin`` (``write_field_serial``, src/field.F90:422-435:
  one Fortran unformatted sequential record of w(1:nv, 1:nx, 1:ny, 1:nz), the
  variable index fastest) or ``rst.bin`` (``write_field``, src/field.F90:437-477: nv
  consecutive global blocks w(l, 1:nx, 1:ny, 1:nz), i fastest, native doubles,
  no record markers), and ``field_info{1,0}.dat`` (``write_field_info``,
  src/multideal/multideal.F90:2440-2470, a one-section cfg file);

and ``run`` is the reference's integration loop (``run``, multideal_gpu.F90:1659-1851)
with those outputs.  Fields are copied from the device only when a file is due.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import struct
import time as _time
from typing import Optional

import numpy as np

from .native import check


# ------------------------------------------------------------------ Fortran edit descriptors
def fortran_es(v: float, w: int = 20, d: int = 10) -> str:
    """ESw.d: one significant digit before the point, d after, exponent 'E+dd'
    (three-digit exponents drop the 'E', as Fortran does), right-justified in w."""
    v = float(v)
    if not math.isfinite(v):
        return ("NaN" if math.isnan(v) else ("-Infinity" if v < 0 else "Infinity")).rjust(w)
    s = f"{v:.{d}E}"
    mant, ex = s.split("E")
    e = int(ex)
    es = f"E{e:+03d}" if abs(e) < 100 else f"{e:+04d}"
    out = mant + es
    return out.rjust(w) if len(out) <= w else "*" * w


def fortran_f(v: float, w: int, d: int) -> str:
    s = f"{float(v):.{d}f}"
    return s.rjust(w) if len(s) <= w else "*" * w


def fortran_i(v: int, w: int) -> str:
    s = str(int(v))
    return s.rjust(w) if len(s) <= w else "*" * w


def progress_line(icyc: int, step_time: float, dt: float, time: float, res7) -> str:
    """One line of print_progress: '(1I10,F18.10,20ES20.10)'."""
    return fortran_i(icyc, 10) + fortran_f(step_time, 18, 10) + "".join(
        fortran_es(v) for v in (dt, time) + tuple(res7))


def es_rows(cols) -> str:
    """Rows of '(nES20.10)' from equal-length columns."""
    cols = [np.asarray(c, float).ravel() for c in cols]
    return "".join("".join(fortran_es(c[i]) for c in cols) + "\n" for i in range(len(cols[0])))


# ------------------------------------------------------------------ example outputs
def write_output_1d(path: str, case, w_aux: np.ndarray):
    """output_1d_*micro_s.dat of the reactive shock tube (multideal_gpu.F90:2540-2548):
    x(i), T, u, w_aux(i,1,1,3) (the third species' mass fraction), '(4ES20.10)'."""
    ng, nx = case.ng, case.nx
    row = lambda j: w_aux[j, ng, ng, ng:ng + nx]
    with open(path, "w") as fh:
        fh.write(es_rows([case.x[ng:ng + nx], row(case.J("T")), row(case.J("U")), row(2)]))


def write_output_lpf(path: str, case, w_aux: np.ndarray):
    """output_LPF.dat of the premixed flame (multideal_gpu.F90:2550-2562): x, T, rho,
    Y_1, Y_4, Y_5, Y_2 (H2, O, OH, H in the flame mechanism's order), '(7ES20.10)'."""
    ng, nx = case.ng, case.nx
    row = lambda j: w_aux[j, ng, ng, ng:ng + nx]
    with open(path, "w") as fh:
        fh.write(es_rows([case.x[ng:ng + nx], row(case.J("T")), row(case.J("R")), row(0), row(3), row(4), row(1)]))


def append_output_batch(path: str, time: float, rho: float, T: float):
    """One line of output_batch.dat (multideal_gpu.F90:2519-2525): time, rho, T of
    cell (1,1,1), '(3ES20.10)'; the reference keeps the unit open, so lines add up."""
    with open(path, "a") as fh:
        fh.write(fortran_es(time) + fortran_es(rho) + fortran_es(T) + "\n")


# ------------------------------------------------------------------ restart
def _interior_vfirst(case, w: np.ndarray) -> np.ndarray:
    """w(1:nv, 1:nx, 1:ny, 1:nz) in Fortran order (variable fastest) from the
    solver's (nv, nzg, nyg, nxg) ghosted array."""
    ng = case.ng
    wi = w[:, ng:ng + case.nz, ng:ng + case.ny, ng:ng + case.nx]      # (nv, nz, ny, nx)
    return np.ascontiguousarray(np.transpose(wi, (1, 2, 3, 0)))          # (nz, ny, nx, nv): nv fastest


def restart_serial_name(ncoords=(0, 0, 0), prefix="rst1") -> str:
    return f"{prefix}_{ncoords[0]:04d}_{ncoords[1]:04d}_{ncoords[2]:04d}.bin"


def write_restart_serial(path: str, case, w: np.ndarray):
    """write_field_serial: one unformatted sequential record (4-byte length markers,
    native byte order) of w(1:nv, 1:nx, 1:ny, 1:nz)."""
    data = _interior_vfirst(case, w).tobytes()
    if len(data) > 2 ** 31 - 1:
        raise ValueError("record longer than 2^31-1 bytes: use the rst.bin form (io_type_w = 2)")
    mark = struct.pack("=i", len(data))
    with open(path, "wb") as fh:
        fh.write(mark)
        fh.write(data)
        fh.write(mark)


def read_restart_serial(path: str, case) -> np.ndarray:
    """read_field_serial: the interior of w as (nv, nz, ny, nx)."""
    nv, n = case.nv, case.nx * case.ny * case.nz
    with open(path, "rb") as fh:
        (ln,) = struct.unpack("=i", fh.read(4))
        if ln != nv * n * 8:
            raise ValueError(f"{path}: record of {ln} bytes, expected {nv * n * 8}")
        a = np.frombuffer(fh.read(ln), dtype=np.float64)
        (ln2,) = struct.unpack("=i", fh.read(4))
        if ln2 != ln:
            raise ValueError(f"{path}: trailing record marker {ln2} != {ln}")
    return np.transpose(a.reshape(case.nz, case.ny, case.nx, nv), (3, 0, 1, 2))


def write_restart_mpiio(path: str, case, w: np.ndarray):
    """write_field on one process: nv consecutive blocks w(l, 1:nx, 1:ny, 1:nz), i
    fastest, native doubles."""
    ng = case.ng
    wi = np.ascontiguousarray(w[:, ng:ng + case.nz, ng:ng + case.ny, ng:ng + case.nx])
    with open(path, "wb") as fh:
        fh.write(wi.tobytes())


def read_restart_mpiio(path: str, case) -> np.ndarray:
    a = np.fromfile(path, dtype=np.float64)
    n = case.nv * case.nx * case.ny * case.nz
    if a.size != n:
        raise ValueError(f"{path}: {a.size} doubles, expected {n}")
    return a.reshape(case.nv, case.nz, case.ny, case.nx)


FIELD_INFO_KEYS = ("icyc0", "time0", "itav", "itslice_vtr", "time_from_last_rst", "time_from_last_write",
                   "time_from_last_stat", "time_from_last_slice", "time_from_last_slice_vtr", "istore")


def write_field_info(path: str, info: dict):
    """write_field_info: '[field_info]' and 'key = value' lines (cfgio, one section)."""
    with open(path, "w") as fh:
        fh.write("[field_info]\n")
        for k in FIELD_INFO_KEYS:
            v = info.get(k, 0)
            fh.write(f"{k} = {v:.17E}\n" if isinstance(v, float) else f"{k} = {int(v)}\n")


def read_field_info(path: str) -> dict:
    from .case import Config
    cfg = Config.from_file(path)
    out = {}
    for k in FIELD_INFO_KEYS:
        if cfg.has_key("field_info", k):
            out[k] = cfg.get("field_info", k, kind=float if k.startswith("time") else int)
    if "time_from_last_slice_vtr" not in out and "time_from_last_slice" in out:
        out["time_from_last_slice_vtr"] = out["time_from_last_slice"]
    return out


# ------------------------------------------------------------------ the run loop
class RunState:
    """The bookkeeping of equation_base the outputs need (field_info keys)."""

    def __init__(self):
        self.icyc0 = 0
        self.itav = 0
        self.itslice_vtr = 0
        self.time_from_last_rst = 0.0
        self.time_from_last_write = 0.0
        self.time_from_last_stat = 0.0
        self.time_from_last_slice = 0.0
        self.time_from_last_slice_vtr = 0.0
        self.istore = 1
        self.done = [0, 0, 0, 0]      # the saved done1..3 of manage_output (and the flame's done1)

    def info(self, icyc, time):
        d = {k: getattr(self, k) for k in FIELD_INFO_KEYS if hasattr(self, k)}
        d["icyc0"] = icyc
        d["time0"] = float(time)
        return d


def compute_residual(sol) -> list:
    """compute_residual (multideal_gpu.F90:1585-1615) through stx_compute_residual."""
    out = (C.c_double * 7)()
    check(sol.lib.stx_compute_residual(sol.ctx, sol.stream, C.c_void_p(sol.fln.data_ptr()),
                                       C.c_void_p(sol.w_aux.data_ptr()), None, sol.dt, out), "compute_residual")
    return list(out)


def manage_output(sol, st: RunState, outdir: str, dtsave_restart: float = 1e30, io_type_w: int = 1):
    """The parts of manage_output (multideal_gpu.F90:2437-2755) on this path: the
    example outputs of flow_init 8 / 9 / 10 and the periodic restart."""
    case, time = sol.case, sol.time
    fi = case.flow_init
    if fi == 8:
        n = int(round(time / sol.dt)) if sol.dt else 0
        if n >= 10 and n % 10 == 0:
            wa = sol.host_w_aux()
            ng = case.ng
            append_output_batch(os.path.join(outdir, "output_batch.dat"), time, wa[case.J("R"), ng, ng, ng],
                                wa[case.J("T"), ng, ng, ng])
    elif fi == 9:
        name = None
        if time >= 170e-6 and st.done[0] == 0:
            name, st.done[0] = "output_1d_170micro_s.dat", 1
        elif time >= 190e-6 and st.done[1] == 0:
            name, st.done[1] = "output_1d_190micro_s.dat", 1
        elif time >= 230e-6 and st.done[2] == 0:
            name, st.done[2] = "output_1d_230micro_s.dat", 1
        if name:
            write_output_1d(os.path.join(outdir, name), case, sol.host_w_aux())
            st.time_from_last_write = 0.0
            st.istore += 1
    elif fi == 10:
        if time >= 1e-3 and st.done[3] == 0:
            st.done[3] = 1
            write_output_lpf(os.path.join(outdir, "output_LPF.dat"), case, sol.host_w_aux())
    st.time_from_last_rst += sol.dt
    if st.time_from_last_rst >= dtsave_restart:
        write_restart(sol, st, outdir, io_type_w)
        st.time_from_last_rst = 0.0


def write_restart(sol, st: RunState, outdir: str, io_type_w: int = 1):
    """copy_gpu_cpu + write_field_serial / write_field + write_field_info."""
    w = sol.host_w()
    if io_type_w == 1:
        write_restart_serial(os.path.join(outdir, restart_serial_name()), sol.case, w)
        write_field_info(os.path.join(outdir, "field_info1.dat"), st.info(sol.icyc, sol.time))
    else:
        write_restart_mpiio(os.path.join(outdir, "rst.bin"), sol.case, w)
        write_field_info(os.path.join(outdir, "field_info0.dat"), st.info(sol.icyc, sol.time))


def read_restart(sol, indir: str, io_type_r: int = 1) -> RunState:
    """restart_type 1 (multideal.F90 initialize -> read_field_serial / read_field and
    read_field_info): the interior of w from rst0_0000_0000_0000.bin (or rst.bin)
    and the loop state from field_info0.dat.  The ghosts are filled by the first
    update_ghost of the run."""
    import torch
    case = sol.case
    if io_type_r == 1:
        wi = read_restart_serial(os.path.join(indir, restart_serial_name(prefix="rst0")), case)
    else:
        wi = read_restart_mpiio(os.path.join(indir, "rst.bin"), case)
    ng = case.ng
    sl = (slice(None), slice(ng, ng + case.nz), slice(ng, ng + case.ny), slice(ng, ng + case.nx))
    sol.w[sl] = torch.from_numpy(np.ascontiguousarray(wi)).to(sol.w.device)
    info = read_field_info(os.path.join(indir, "field_info0.dat"))
    st = RunState()
    for k, v in info.items():
        setattr(st, k, v)
    sol.icyc = int(info.get("icyc0", 0))
    sol.time = float(info.get("time0", 0.0))
    st.icyc0 = sol.icyc
    return st


def run(sol, num_iter: int, outdir: Optional[str] = None, print_control: int = 1000, io_type_w: int = 1,
        dtsave_restart: float = 1e30, state: Optional[RunState] = None, progress=print,
        t_end: Optional[float] = None):
    """The reference's run loop (multideal_gpu.F90:1687-1851) on a Solver: prepare,
    num_iter steps with the residual and progress line every print_control steps
    (progress.out in outdir), the example outputs of manage_output, and the final
    restart and field_info.  t_end: also stop after the first step that reaches
    this time.  Returns the progress rows."""
    import torch
    st = state or RunState()
    st.icyc0 = sol.icyc
    if outdir:
        os.makedirs(outdir, exist_ok=True)
    sol.prepare()
    rows = []
    pfh = open(os.path.join(outdir, "progress.out"), "a") if outdir else None
    try:
        for _ in range(num_iter):
            t0 = _time.perf_counter()
            sol.icyc += 1
            if (sol.icyc - st.icyc0) % sol.case.iter_dt_recompute == 0:
                sol.compute_aux(1, 0)
                sol.compute_dt()
            sol.advance_solution()
            sol.compute_aux(1, 0)
            res = None
            if (sol.icyc - st.icyc0) % print_control == 0:
                res = compute_residual(sol)
                if math.isnan(res[0]):
                    raise FloatingPointError(f"BOOM: residual is NaN at step {sol.icyc}")
            sol.time = sol.time + sol.dt
            if outdir:
                manage_output(sol, st, outdir, dtsave_restart, io_type_w)
            if res is not None:
                torch.cuda.synchronize(sol.device)
                line = progress_line(sol.icyc, _time.perf_counter() - t0, sol.dt, sol.time, res)
                rows.append([sol.icyc, sol.dt, sol.time] + res)
                if pfh:
                    pfh.write(line + "\n")
                if progress:
                    progress(line)
            if t_end is not None and sol.time >= t_end:
                break
        if outdir:
            write_restart(sol, st, outdir, io_type_w)
    finally:
        if pfh:
            pfh.close()
    return rows
