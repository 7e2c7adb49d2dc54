"""Case set-up: the host side of the reference's ``equation_multideal`` initialisation.

Mirrors, for the hot-path subset, ``initialize`` (src/multideal/multideal.F90:432-974):
INI keys, grid generation and metrics (src/grid.F90:56-133, 569-627,
src/field.F90:300-347), reference state and ``set_flow_params`` (:3415-3539),
``bc_preproc`` (:5671-5718), ``runge_kutta_initialize`` (:5763-5786) and the
initial conditions used by the examples (``initial_conditions`` :3698-3742,
``init_reactor`` :5608-5669, ``init_reactive_tube`` :5305-5381).  Options that
belong to subsystems outside this path (IBM, LES, recycling, NR boundaries,
non-uniform grids) are rejected with an error, as ``fail_input_any`` would.

Field arrays are numpy arrays in the reference's SoA Fortran order, stored as
C-order arrays of shape (nvar, nzg, nyg, nxg); element [m, k+ng-1, j+ng-1, i+ng-1]
is the Fortran w(i, j, k, m+1).
"""
from __future__ import annotations

import ctypes as C
import math
import re
from typing import Dict, Optional

import numpy as np

from . import mech as M
from .native import StxGrid, StxParams, StxTables

TOL_ITER = 1e-9        # src/parameters.F90:49
# ghost-fill tags of update_ghost on this path (multideal_gpu.F90:1176-1233): 0 periodic,
# 1 free stream, 2 extrapolation, 4 subsonic extrapolation at p0, 5 symmetry,
# 6 isothermal wall, 7 open outflow, 8 adiabatic wall
BC_TAGS = (0, 1, 2, 4, 5, 6, 7, 8)
TOL_ITER_NR = 1e-12    # src/parameters.F90:50

# deriv coefficients (grid.F90:135-182)
_CD1 = {1: [0.5], 2: [2.0 / 3.0, -1.0 / 12.0], 3: [0.75, -0.15, 1.0 / 60.0],
        4: [4.0 / 5.0, -1.0 / 5.0, 4.0 / 105.0, -1.0 / 280.0]}


class Config:
    """Reader for ``multideal.ini`` (cfgio syntax: [section], key = value ; comment)."""

    def __init__(self, text: str = ""):
        self.data: Dict[str, Dict[str, str]] = {}
        sec = None
        for raw in text.splitlines():
            line = raw.split(";", 1)[0].strip()
            if not line:
                continue
            m = re.match(r"^\[(.+)\]$", line)
            if m:
                sec = m.group(1).strip()
                self.data.setdefault(sec, {})
                continue
            if "=" in line and sec is not None:
                k, v = line.split("=", 1)
                self.data[sec][k.strip()] = v.strip()

    @classmethod
    def from_file(cls, path: str) -> "Config":
        with open(path) as fh:
            return cls(fh.read())

    def has_key(self, sec: str, key: str) -> bool:
        return sec in self.data and key in self.data[sec]

    def get(self, sec: str, key: str, default=None, kind=float):
        if not self.has_key(sec, key):
            if default is None:
                raise KeyError(f"missing key [{sec}] {key}")
            return default
        v = self.data[sec][key]
        if kind is int:
            return int(float(v))
        if kind is float:
            return float(v.replace("D", "E").replace("d", "e"))
        return v

    def set(self, sec: str, key: str, value):
        self.data.setdefault(sec, {})[key] = str(value)


class Case:
    """Everything the kernels need for one solve, on the host."""

    def __init__(self, cfg: Config, tables: M.Tables, init_Y: Optional[np.ndarray] = None, alloc_fields: bool = True):
        self.cfg = cfg
        self.tb = tables
        ns = tables.ns
        self.ns = ns
        self.nv = ns + 4
        # --- boundary conditions and periodicity (multideal.F90:491-517)
        keys = ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
        self.bctags = [cfg.get("bc", k, kind=int) for k in keys]
        self.bctags_nr = [cfg.get("bc", k + "_nr", 0, kind=int) for k in keys]
        self.periodic = [False] * 3
        for d in range(3):
            if 0 in self.bctags[2 * d: 2 * d + 2]:
                self.bctags[2 * d] = self.bctags[2 * d + 1] = 0
                self.periodic[d] = True
        for t in self.bctags:
            if t not in BC_TAGS:
                raise ValueError(f"bc tag {t} is outside the supported path {sorted(BC_TAGS)} "
                                 "(9 laminar-profile inflow, 10 recycling, 26/28 jets, 46/56 special walls are not)")
        for t in self.bctags_nr:
            if t not in (0, 1, 2, 3, 6):
                raise ValueError(f"bc *_nr = {t}: the characteristic treatment takes 0, 1, 2, 3 or 6")
        # --- grid (uniform only)
        gtype = cfg.get("grid", "grid_type", kind=int)
        if gtype != 2:
            raise ValueError("only grid_type = 2 (uniform) is supported")
        self.nx = cfg.get("grid", "nxmax", kind=int)
        self.ny = cfg.get("grid", "nymax", kind=int)
        self.nz = cfg.get("grid", "nzmax", kind=int)
        self.ng = cfg.get("grid", "ng", kind=int)
        dom = [cfg.get("grid", "domain_size_" + a) for a in "xyz"]
        morder = cfg.get("grid", "metrics_order", kind=int)
        self.ep_order = cfg.get("numerics", "ep_order", kind=int)
        self._make_grid(dom, morder)
        # --- numerics
        self.nkeep = cfg.get("numerics", "nkeep", 0, kind=int)
        self.weno_scheme = cfg.get("numerics", "weno_scheme", kind=int)
        self.weno_version = cfg.get("numerics", "weno_version", kind=int)
        self.flux_splitting = cfg.get("numerics", "flux_splitting", 0, kind=int)
        self.visc_order = self.ep_order           # multideal.F90:683-686
        self.conservative_viscous = cfg.get("numerics", "conservative_viscous", kind=int)
        if self.conservative_viscous != 1:
            raise ValueError("conservative_viscous = 0 (Laplacian form) is not on this path")
        self.sensor_threshold = cfg.get("numerics", "sensor_threshold")
        self.sensor_type = cfg.get("numerics", "sensor_type", 1, kind=int)
        rk_type = cfg.get("numerics", "rk_type", 1, kind=int)
        if rk_type != 1:
            raise ValueError("only rk_type = 1 (Wray RK3) is supported")
        self.rhork = [0.0, -17.0 / 60.0, -5.0 / 12.0]
        self.gamrk = [8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0]
        # --- chemistry
        self.enable_chemistry = cfg.get("fluid", "enable_chemistry", 0, kind=int)
        self.rosenbrock_version = cfg.get("numerics", "rosenbrock_version", 2, kind=int)
        self.operator_splitting = cfg.get("numerics", "operator_splitting", 2, kind=int)
        if self.enable_chemistry == 2:
            if self.rosenbrock_version == 1 and self.operator_splitting == 1:
                raise ValueError("operator_splitting 1 not implement for rosenbrock_version 1")
        self.ros_eps = cfg.get("numerics", "ros_eps", 1e-8)
        self.ros_maxsteps = cfg.get("numerics", "ros_maxsteps", 10000, kind=int)
        self.ros_maxtry = cfg.get("numerics", "ros_maxtry", 40, kind=int)
        self.cfl = cfg.get("controls", "cfl")
        self.num_iter = cfg.get("controls", "num_iter", 0, kind=int)
        self.iter_dt_recompute = cfg.get("controls", "iter_dt_recompute", 1, kind=int)
        self.flow_init = cfg.get("flow", "flow_init", kind=int)
        if cfg.get("lespar", "enable_les", 0, kind=int) > 0:
            raise ValueError("LES is not on this path")
        self.nv_aux = 2 * ns + 13 + (2 * (ns + 1) if self.enable_chemistry > 0 else 0)
        # --- reference state (multideal.F90:2817-2850) and flow parameters (:3415-3539)
        if init_Y is None:
            init_Y = np.array([cfg.get("ref_state", f"init_Y_{k + 1:02d}") for k in range(ns)])
        self.init_Y = np.asarray(init_Y, float)
        self.rmixt0 = float(np.dot(tables.rgas, self.init_Y))
        rg = self.rmixt0
        have = {k: cfg.has_key("ref_state", k) for k in ("t0", "p0", "rho0")}
        if not have["t0"] and have["p0"] and have["rho0"]:
            self.p0 = cfg.get("ref_state", "p0"); self.rho0 = cfg.get("ref_state", "rho0")
            self.t0 = self.p0 / self.rho0 / rg
        elif not have["p0"] and have["t0"] and have["rho0"]:
            self.t0 = cfg.get("ref_state", "t0"); self.rho0 = cfg.get("ref_state", "rho0")
            self.p0 = self.rho0 * rg * self.t0
        elif not have["rho0"] and have["t0"] and have["p0"]:
            self.t0 = cfg.get("ref_state", "t0"); self.p0 = cfg.get("ref_state", "p0")
            self.rho0 = self.p0 / rg / self.t0
        else:
            raise ValueError("Problem with the reference state")
        self.cp0 = M.mixture_cp(tables, self.t0, self.init_Y)
        self.gam = self.cp0 / (self.cp0 - rg)
        self.p0 = self.rho0 * rg * self.t0
        self.c0 = math.sqrt(self.gam * rg * self.t0)
        self.u0 = cfg.get("ref_state", "u0", 0.0)
        e0 = M.mixture_e(tables, self.t0, self.init_Y)
        self.winf = np.zeros(self.nv)
        self.winf[:ns] = self.rho0 * self.init_Y
        self.winf[ns] = self.rho0 * self.u0
        self.winf[ns + 3] = self.rho0 * (e0 + 0.5 * self.u0 ** 2)
        if abs(self.u0) < TOL_ITER:
            self.u0 = self.c0
        self.eps_sensor = self.u0 ** 2
        # --- bc_preproc (multideal.F90:5671-5718): a face with a characteristic
        # treatment leaves its boundary cells out of the convective flux
        # divergence (bc_nr supplies their convective term)
        self.force_zero_flux = [0] * 6
        self.eul = [1, self.nx, 1, self.ny, 1, self.nz]
        for ilat in range(6):
            if self.bctags_nr[ilat] != 0:
                self.eul[ilat] += 1 if ilat % 2 == 0 else -1
        self.T_wall = cfg.get("flow", "T_wall", 0.0) if cfg.has_key("flow", "T_wall") else self.t0
        # --- fields
        self.nxg, self.nyg, self.nzg = self.nx + 2 * self.ng, self.ny + 2 * self.ng, self.nz + 2 * self.ng
        self._keep = []
        self.fluid_mask = None
        if not alloc_fields:      # fields are built on the device by the caller
            self.w = self.w_aux = None
            return
        self.w = np.empty((self.nv, self.nzg, self.nyg, self.nxg))
        for m in range(self.nv):
            self.w[m] = self.winf[m]
        self.w_aux = np.zeros((self.nv_aux, self.nzg, self.nyg, self.nxg))
        self.w_aux[ns + 4] = self.t0                  # J_T initial guess (multideal.F90:3706)
        self.fluid_mask = None
        self._keep = []
        if self.flow_init == 8:
            self._init_reactor()
        elif self.flow_init == 9:
            self._init_reactive_tube()
        elif self.flow_init in (-1,):
            pass
        elif self.flow_init == 10:
            pass    # init_premix: the profile comes from premix.dat (init_premix below)
        elif self.flow_init == 100:
            pass    # caller-provided field (synthetic cases)
        else:
            raise ValueError(f"flow_init {self.flow_init} is not supported on this path")

    # ------------------------------------------------------------------ grid
    def _make_grid(self, dom, morder):
        ng = self.ng
        self.xg = []
        for d, n in enumerate((self.nx, self.ny, self.nz)):
            L = dom[d]
            dx = L / (n - 1) if n > 1 else L
            if self.periodic[d] or n == 1:
                dx = L / n
            if n > 1 and not self.periodic[d]:
                dx = L / (n - 1)
            # x has one extra node (grid.F90:580-582)
            top = n + ng + 1 if d == 0 else n + ng
            idx = np.arange(1 - ng, top + 1)
            self.xg.append((idx - 1) * dx)
        mm = morder // 2
        c = _CD1[mm]
        met = []
        for d, n in enumerate((self.nx, self.ny, self.nz)):
            xg = self.xg[d]
            dxg = np.zeros(n)
            for i in range(1, n + 1):
                s = 0.0
                for l in range(1, mm + 1):
                    s = s + c[l - 1] * (xg[i + l + ng - 1] - xg[i - l + ng - 1])
                dxg[i - 1] = s
            met.append(dxg)
        self.x = np.ascontiguousarray(self.xg[0][: self.nx + 2 * ng])
        self.y = np.ascontiguousarray(self.xg[1][: self.ny + 2 * ng])
        self.z = np.ascontiguousarray(self.xg[2][: self.nz + 2 * ng])
        self.dcsidx = 1.0 / met[0]
        self.detady = 1.0 / met[1]
        self.dzitdz = 1.0 / met[2]
        self.dcsidxs = self.dcsidx * self.dcsidx
        self.detadys = self.detady * self.detady
        self.dzitdzs = self.dzitdz * self.dzitdz

    # ------------------------------------------------------------------ ICs
    def _cons(self, rho, u, T, Y):
        w = np.zeros(self.nv)
        w[: self.ns] = rho * Y
        w[self.ns] = rho * u
        w[self.ns + 3] = rho * (M.mixture_e(self.tb, T, Y) + 0.5 * u * u)
        return w

    def _init_reactor(self):
        rho = self.p0 / np.dot(self.tb.rgas, self.init_Y) / self.t0
        wr = self._cons(rho, 0.0, self.t0, self.init_Y)
        ng = self.ng
        self.w[:, ng:ng + self.nz, ng:ng + self.ny, ng:ng + self.nx] = wr[:, None, None, None]

    def _init_reactive_tube(self, rho_t=0.18075, u_t=-487.34, p_t=35594.0):
        rm = np.dot(self.tb.rgas, self.init_Y)
        t_t = p_t / rm / rho_t
        wt = self._cons(rho_t, u_t, t_t, self.init_Y)
        ng = self.ng
        x = self.x
        for i in range(1, self.nx + 1):
            if x[i + ng - 1] >= 0.5 * x[self.nx + ng - 1]:
                self.w[:, ng:ng + self.nz, ng:ng + self.ny, i + ng - 1] = wt[:, None, None]

    def init_premix(self, u, T, Y):
        """init_premix (multideal.F90:5534-5606): the 1-D profile of premix.dat (per
        cell i: u, T, Y_1..Y_ns) on every (j, k) line, at the reference pressure.
        As in the reference, the mixture gas constant and rho*Y_k use the file's
        mass fractions as they are, while the internal energy is evaluated with
        |Y_k| < 1e-25 set to zero."""
        u, T = np.asarray(u, float)[: self.nx], np.asarray(T, float)[: self.nx]
        Y = np.asarray(Y, float)[:, : self.nx]
        rm = np.einsum("k,kx->x", self.tb.rgas, Y)
        Yc = np.where(np.abs(Y) < 1e-25, 0.0, Y)
        rho = self.p0 / rm / T
        e = mixture_e_field(self.tb, T, Yc)
        ng, ns = self.ng, self.ns
        sl = (slice(ng, ng + self.nz), slice(ng, ng + self.ny), slice(ng, ng + self.nx))
        self.w[(slice(0, ns),) + sl] = (rho[None, :] * Y)[:, None, None, :]
        self.w[(ns,) + sl] = (rho * u)[None, None, :]
        self.w[(ns + 1,) + sl] = 0.0
        self.w[(ns + 2,) + sl] = 0.0
        self.w[(ns + 3,) + sl] = (rho * (e + 0.5 * u * u))[None, None, :]

    def set_interior(self, rho, u, v, w, T, Y):
        """Set the interior from primitive fields of shape (nz, ny, nx) (Y: (ns, nz, ny, nx))."""
        ng, ns = self.ng, self.ns
        sl = (slice(ng, ng + self.nz), slice(ng, ng + self.ny), slice(ng, ng + self.nx))
        e = mixture_e_field(self.tb, T, Y)
        self.w[(slice(0, ns),) + sl] = rho[None] * Y
        self.w[(ns,) + sl] = rho * u
        self.w[(ns + 1,) + sl] = rho * v
        self.w[(ns + 2,) + sl] = rho * w
        self.w[(ns + 3,) + sl] = rho * (e + 0.5 * (u * u + v * v + w * w))
        self.w_aux[(ns + 4,) + sl] = T

    # ------------------------------------------------------------------ structs
    def _p(self, a, ctype=C.c_double):
        a = np.ascontiguousarray(a)
        self._keep.append(a)
        return a.ctypes.data_as(C.POINTER(ctype))

    def params_struct(self) -> StxParams:
        p = StxParams()
        p.nv_aux = self.nv_aux
        p.p0, p.rho0, p.u0, p.eps_sensor, p.tol_iter_nr = self.p0, self.rho0, self.u0, self.eps_sensor, TOL_ITER_NR
        p.ep_order, p.nkeep, p.weno_scheme, p.weno_version = self.ep_order, self.nkeep, self.weno_scheme, self.weno_version
        p.flux_splitting, p.sensor_type, p.visc_order = self.flux_splitting, self.sensor_type, self.visc_order
        p.conservative_viscous = self.conservative_viscous
        p.sensor_threshold = self.sensor_threshold
        for q in range(6):
            p.bctags[q] = self.bctags[q]
            p.bctags_nr[q] = self.bctags_nr[q]
            p.force_zero_flux[q] = self.force_zero_flux[q]
        p.eul_imin, p.eul_imax, p.eul_jmin, p.eul_jmax, p.eul_kmin, p.eul_kmax = self.eul
        p.enable_chemistry = self.enable_chemistry
        p.rosenbrock_version = self.rosenbrock_version
        p.operator_splitting = self.operator_splitting
        p.ros_maxsteps, p.ros_maxtry, p.ros_eps = self.ros_maxsteps, self.ros_maxtry, self.ros_eps
        p.nrk = 3
        for q in range(3):
            p.rhork[q] = self.rhork[q]
            p.gamrk[q] = self.gamrk[q]
        p.winf = self._p(self.winf)
        p.T_wall = self.T_wall
        return p

    def tables_struct(self) -> StxTables:
        tb = self.tb
        t = StxTables()
        t.ns, t.nr = tb.ns, tb.nr
        t.indx_cp_l, t.indx_cp_r, t.nsetcv, t.num_t_tab = tb.indx_cp_l, tb.indx_cp_r, tb.nsetcv, tb.num_t_tab
        t.t_min_tab, t.dt_tab, t.R_univ = tb.t_min_tab, tb.dt_tab, M.R_UNIV
        F = lambda a: self._p(np.asarray(a, float).ravel(order="F"))
        I = lambda a: self._p(np.asarray(a, np.int32).ravel(order="F"), C.c_int32)
        t.mw, t.mwinv, t.rgas = F(tb.mw), F(1.0 / tb.mw), F(tb.rgas)
        t.trange, t.cp_coeff, t.cv_coeff = F(tb.trange), F(tb.cp_coeff), F(tb.cv_coeff)
        t.visc, t.lam, t.diffbin = F(tb.visc), F(tb.lam), F(tb.diffbin)
        nr = max(tb.nr, 1)
        t.reac_ty = I(tb.reac_ty if tb.nr else np.zeros(1))
        t.is_rev = I(tb.is_rev if tb.nr else np.zeros(1))
        z2 = np.zeros((nr, 2))
        t.arr_a = F(tb.arr_a if tb.nr else z2)
        t.arr_b = F(tb.arr_b if tb.nr else z2)
        t.arr_ea = F(tb.arr_ea if tb.nr else z2)
        t.falloff = F(tb.falloff if tb.nr else np.zeros((nr, 5)))
        zs = np.zeros((nr, tb.ns))
        t.tb_eff = F(tb.tb_eff if tb.nr else zs)
        t.r_coeffs = F(tb.r_coeffs if tb.nr else zs)
        t.p_coeffs = F(tb.p_coeffs if tb.nr else zs)
        t.kc_tab = F(tb.kc_tab if tb.nr else np.zeros((tb.num_t_tab + 1, 1)))
        t.n_eoi = 1
        t.aw_eoi, t.coeff_eoi, t.beta0 = F(np.ones(1)), F(np.ones(1)), F(np.array([1.0, 0.0]))
        t.nainsp = I(np.zeros(tb.ns))
        return t

    def grid_struct(self) -> StxGrid:
        g = StxGrid()
        g.nx, g.ny, g.nz, g.ng = self.nx, self.ny, self.nz, self.ng
        g.x, g.y, g.z = self._p(self.x), self._p(self.y), self._p(self.z)
        g.dcsidx, g.detady, g.dzitdz = self._p(self.dcsidx), self._p(self.detady), self._p(self.dzitdz)
        g.dcsidxs, g.detadys, g.dzitdzs = self._p(self.dcsidxs), self._p(self.detadys), self._p(self.dzitdzs)
        return g

    # ------------------------------------------------------------------ helpers
    def J(self, name: str) -> int:
        """0-based w_aux slot of a J_* name (index_define.h)."""
        off = {"U": 1, "V": 2, "W": 3, "H": 4, "T": 5, "P": 6, "C": 7, "MU": 8, "DUC": 9, "DIV": 10,
               "R": 11, "Z": 12, "K_COND": 13}
        return self.ns + off[name] - 1

    def interior(self, a):
        ng = self.ng
        return a[..., ng:ng + self.nz, ng:ng + self.ny, ng:ng + self.nx]


def mixture_e_field(tb: M.Tables, T: np.ndarray, Y: np.ndarray) -> np.ndarray:
    """Vectorised ``get_e_from_temperature`` (per-species NASA range by locate)."""
    e = np.zeros_like(T)
    icl, icr = tb.indx_cp_l, tb.indx_cp_r
    for k in range(tb.ns):
        rng = np.ones(T.shape, int)
        if tb.nsetcv > 1:
            jl = np.zeros(T.shape, int)
            for jm in range(1, tb.nsetcv + 2):
                jl = np.where(T >= tb.trange[k, jm - 1], jm, jl)
            rng = np.clip(jl, 1, tb.nsetcv)
        ek = np.zeros_like(T)
        for m in range(1, tb.nsetcv + 1):
            cvc = tb.cv_coeff[:, k, m - 1]
            em = np.full_like(T, cvc[icr + 1 - icl])
            for l in range(icl, icr + 1):
                if l == -1:
                    em = em + cvc[l - icl] * np.log(T)
                else:
                    em = em + cvc[l - icl] / (l + 1.0) * T ** (l + 1)
            ek = np.where(rng == m, em, ek)
        e = e + ek * Y[k]
    return e


def read_premix(path: str, ns: int):
    """The reference's premix.dat (one line per cell: x, u, T, Y_1..Y_ns) as arrays
    x, u, T (n) and Y (ns, n)."""
    a = np.loadtxt(path, ndmin=2)
    if a.shape[1] != 3 + ns:
        raise ValueError(f"{path}: {a.shape[1]} columns, expected {3 + ns}")
    return a[:, 0], a[:, 1], a[:, 2], a[:, 3:].T.copy()


def default_ini(nx, ny, nz, L=(1.0, 1.0, 1.0), bc=(0, 0, 0, 0, 0, 0), t0=1000.0, p0=101325.0,
                Y=None, ns=9, chemistry=2, rosenbrock_version=2, splitting=2, weno_version=1,
                sensor_threshold=0.1, sensor_type=1, nkeep=1, ep_order=6, flux_splitting=0,
                cfl=0.5, flow_init=100, weno_scheme=3, ng=3, bc_nr=(0, 0, 0, 0, 0, 0),
                T_wall=None) -> Config:
    """A Config with the keys the solver reads, for synthetic cases."""
    cfg = Config()
    cfg.set("ref_state", "t0", t0); cfg.set("ref_state", "p0", p0); cfg.set("ref_state", "u0", 0.0)
    if Y is not None:
        for k, y in enumerate(Y):
            cfg.set("ref_state", f"init_Y_{k + 1:02d}", repr(float(y)))
    for a, n, l in zip("xyz", (nx, ny, nz), L):
        cfg.set("grid", f"n{a}max", n); cfg.set("grid", f"domain_size_{a}", repr(float(l)))
    cfg.set("grid", "ng", ng); cfg.set("grid", "metrics_order", ep_order); cfg.set("grid", "grid_type", 2)
    for k, v, vn in zip(["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"], bc, bc_nr):
        cfg.set("bc", k, v); cfg.set("bc", k + "_nr", vn)
    cfg.set("controls", "cfl", cfl); cfg.set("controls", "num_iter", 1); cfg.set("controls", "iter_dt_recompute", 1)
    for k, v in dict(ep_order=ep_order, nkeep=nkeep, visc_order=ep_order, conservative_viscous=1,
                     weno_scheme=weno_scheme, weno_version=weno_version, flux_splitting=flux_splitting,
                     sensor_threshold=sensor_threshold, sensor_type=sensor_type, rk_type=1,
                     ros_dttry=1e-9, ros_eps=1e-8, ros_maxsteps=10000, ros_maxtry=40,
                     operator_splitting=splitting, rosenbrock_version=rosenbrock_version).items():
        cfg.set("numerics", k, v)
    cfg.set("flow", "flow_init", flow_init)
    if T_wall is not None:
        cfg.set("flow", "T_wall", T_wall)
    cfg.set("fluid", "use_cantera", 1); cfg.set("fluid", "enable_chemistry", chemistry)
    return cfg
