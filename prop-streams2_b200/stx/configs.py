"""Workload builders for the reacting-step configurations.

``turbulence`` is the 3-D periodic reacting decaying-turbulence case: 9-species
H2/air premixture at equivalence ratio 0.7, T = 1000 K, p = 1 atm, random-phase
solenoidal velocity with E(k) ~ k^4 exp(-2 (k/4)^2) rescaled to u_rms = 0.3 c0
(seeded), hybrid WENO5-Z / KEEP(2) fluxes switched by the modified Ducros sensor
(threshold 0.1), mixture-averaged transport, Strang-split ROK4 chemistry.  The
reference ships no initial condition for it; both the GPU solver and the CPU
oracle take the field produced here.

``shock_tube`` is the reference's reactive shock tube (examples/reactive_shock_tube)
on a chosen number of cells.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import case as CS
from . import mech as M

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def mechanism(name: str) -> M.Mechanism:
    with open(os.path.join(DATA, f"mech_{name}.json")) as fh:
        return M.mechanism_from_dict(json.load(fh))


def h2air_Y(phi: float, mech: M.Mechanism) -> np.ndarray:
    X = np.zeros(mech.ns)
    X[mech.index("H2")] = 2.0 * phi
    X[mech.index("O2")] = 1.0
    X[mech.index("N2")] = 3.76
    X /= X.sum()
    mw = np.array([s.mw for s in mech.species])
    Y = X * mw
    return Y / Y.sum()


TURB = dict(T0=1000.0, p0=101325.0, phi=0.7, k0=4.0, mach_rms=0.3, ell=1.0e-3,
            sensor_threshold=0.1, sensor_type=1, nkeep=2, weno_version=1, cfl=0.5)


def turbulence_case(n: int, tables: M.Tables = None, alloc_fields: bool = False, **over):
    """Case object (metadata, tables, grid) of the turbulence workload on an n^3 box
    of side 2*pi*ell; the grid spacing is kept at 2*pi*ell/256 for any n so that a
    smaller box is a same-resolution sample of the 256^3 case."""
    p = dict(TURB)
    p.update(over)
    mech = mechanism("h2air_9sp")
    Y = h2air_Y(p["phi"], mech)
    L = 2.0 * math.pi * p["ell"] * n / 256.0
    cfg = CS.default_ini(n, n, n, L=(L, L, L), bc=(0,) * 6, t0=p["T0"], p0=p["p0"], Y=Y, ns=mech.ns,
                         chemistry=2, rosenbrock_version=2, splitting=2, weno_version=p["weno_version"],
                         sensor_threshold=p["sensor_threshold"], sensor_type=p["sensor_type"], nkeep=p["nkeep"],
                         ep_order=6, flux_splitting=0, cfl=p["cfl"], flow_init=100)
    if tables is None:
        tables = M.build_tables(mech, p["p0"], 200.0, 5500.0, 1.0)
    c = CS.Case(cfg, tables, alloc_fields=alloc_fields)
    c.turb = p
    c.turb_Y = Y
    return c


def turbulence_velocity(n: int, seed: int, k0: float = 4.0, xp=np, device=None):
    """Random-phase solenoidal velocity on an n^3 periodic grid with
    E(k) ~ k^4 exp(-2 (k/k0)^2), unit rms per component (float64).
    xp is numpy or torch (then the field is built on ``device``)."""
    if xp is np:
        rng = np.random.default_rng(seed)
        k1 = np.fft.fftfreq(n, d=1.0 / n)
        kr = np.fft.rfftfreq(n, d=1.0 / n)
        kx = kr[None, None, :]
        ky = k1[None, :, None]
        kz = k1[:, None, None]
        kk = np.sqrt(kx * kx + ky * ky + kz * kz)
        amp = np.zeros_like(kk)
        nz = kk > 0
        amp[nz] = np.sqrt(kk[nz] ** 4 * np.exp(-2.0 * (kk[nz] / k0) ** 2) / (4.0 * np.pi * kk[nz] ** 2))
        comps = []
        for _ in range(3):
            a = (rng.standard_normal(kk.shape) + 1j * rng.standard_normal(kk.shape)) * amp
            comps.append(a)
        kd = np.where(nz, kk * kk, 1.0)
        dot = (kx * comps[0] + ky * comps[1] + kz * comps[2]) / kd
        out = []
        for a, kc in zip(comps, (kx, ky, kz)):
            out.append(np.fft.irfftn(a - kc * dot, s=(n, n, n), axes=(0, 1, 2)))
        return out
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    k1 = torch.fft.fftfreq(n, d=1.0 / n, device=device, dtype=torch.float64)
    kr = torch.fft.rfftfreq(n, d=1.0 / n, device=device, dtype=torch.float64)
    kx = kr[None, None, :]
    ky = k1[None, :, None]
    kz = k1[:, None, None]
    kk = torch.sqrt(kx * kx + ky * ky + kz * kz)
    nzm = kk > 0
    kks = torch.where(nzm, kk, torch.ones_like(kk))
    amp = torch.where(nzm, torch.sqrt(kks ** 4 * torch.exp(-2.0 * (kks / k0) ** 2) / (4.0 * math.pi * kks ** 2)),
                      torch.zeros_like(kk))
    comps = []
    for _ in range(3):
        re = torch.randn(kk.shape, generator=g, device=device, dtype=torch.float64)
        im = torch.randn(kk.shape, generator=g, device=device, dtype=torch.float64)
        comps.append(torch.complex(re, im) * amp)
    kd = torch.where(nzm, kk * kk, torch.ones_like(kk))
    dot = (kx * comps[0] + ky * comps[1] + kz * comps[2]) / kd
    return [torch.fft.irfftn(a - kc * dot, s=(n, n, n)) for a, kc in zip(comps, (kx, ky, kz))]


def turbulence_fields(c, seed: int, xp=np, device=None):
    """Conservative state w and the T guess of the turbulence case (interior and
    ghosts: ghosts are later overwritten by the periodic exchange)."""
    p = c.turb
    tb = c.tb
    Y = c.turb_Y
    n = c.nx
    rm = float(np.dot(tb.rgas, Y))
    rho = p["p0"] / (rm * p["T0"])
    cp = M.mixture_cp(tb, p["T0"], Y)
    c0 = math.sqrt(cp / (cp - rm) * rm * p["T0"])
    e0 = M.mixture_e(tb, p["T0"], Y)
    u, v, w = turbulence_velocity(n, seed, p["k0"], xp=xp, device=device)
    if xp is np:
        rms = np.sqrt((u * u + v * v + w * w).mean() / 3.0)
    else:
        rms = float(((u * u + v * v + w * w).mean() / 3.0).sqrt())
    s = p["mach_rms"] * c0 / rms
    u, v, w = u * s, v * s, w * s
    ng, nv, ns = c.ng, c.nv, c.ns
    shape = (nv, c.nzg, c.nyg, c.nxg)
    if xp is np:
        W = np.zeros(shape)
        WA = np.zeros((c.nv_aux, c.nzg, c.nyg, c.nxg))
    else:
        import torch
        W = torch.zeros(shape, dtype=torch.float64, device=device)
        WA = torch.zeros((c.nv_aux, c.nzg, c.nyg, c.nxg), dtype=torch.float64, device=device)
    # every point, ghost edges and corners included, starts from the mean state
    # (initial_conditions, multideal.F90:3703-3705), then the interior is set
    for k in range(ns):
        W[k] = rho * Y[k]
    W[ns + 3] = rho * e0
    sl = (slice(ng, ng + n),) * 3
    for k in range(ns):
        W[(k,) + sl] = rho * Y[k]
    W[(ns,) + sl] = rho * u
    W[(ns + 1,) + sl] = rho * v
    W[(ns + 2,) + sl] = rho * w
    W[(ns + 3,) + sl] = rho * (e0 + 0.5 * (u * u + v * v + w * w))
    WA[ns + 4] = p["T0"]
    return W, WA


# The reactive shock tube's inputs (examples/reactive_shock_tube/multideal.ini):
# H2:O2:Ar = 2:1:7 by moles, reflecting wall at xmin, extrapolation at xmax,
# WENO5 everywhere (threshold -0.2), Strang + ROK4, fixed dt 2e-8 s.
TUBE_INI = {
    "ref_state": {"rho0": "0.072", "p0": "7173.", "u0": "0.", "init_Y_01": "0.01267282566",
                  "init_Y_02": "0.10138260528", "init_Y_03": "0.", "init_Y_04": "0.", "init_Y_05": "0.",
                  "init_Y_06": "0.", "init_Y_07": "0.", "init_Y_08": "0.", "init_Y_09": "0.88594456906"},
    "grid": {"domain_size_x": "0.12", "domain_size_y": "0.01", "domain_size_z": "0.01", "nymax": "1",
             "nzmax": "1", "ng": "3", "metrics_order": "6", "grid_type": "2"},
    "bc": {"xmin": "8", "xmax": "2", "ymin": "0", "ymax": "0", "zmin": "0", "zmax": "0", "xmin_nr": "0",
           "xmax_nr": "0", "ymin_nr": "0", "ymax_nr": "0", "zmin_nr": "0", "zmax_nr": "0"},
    "controls": {"cfl": "-2E-8", "iter_dt_recompute": "1", "num_iter": "1"},
    "numerics": {"ep_order": "6", "nkeep": "0", "visc_order": "6", "conservative_viscous": "1", "weno_scheme": "3",
                 "weno_version": "1", "flux_splitting": "0", "sensor_threshold": "-0.2", "sensor_type": "0",
                 "rk_type": "1", "ros_dttry": "1.e-9", "ros_eps": "1.e-8", "ros_maxsteps": "10000",
                 "ros_maxtry": "40", "operator_splitting": "2", "rosenbrock_version": "2"},
    "flow": {"flow_init": "9"},
    "fluid": {"use_cantera": "1", "enable_chemistry": "2", "t_min_tab": "200.", "t_max_tab": "20000.",
              "dt_tab": "1."},
}


def tube_case(nx: int, ny: int = 1, tables: M.Tables = None):
    """The reactive shock tube on nx x ny cells (ny > 1: the same 1-D state on a
    2-D periodic-in-y strip of height 0.01 m * ny / 128)."""
    cfg = CS.Config()
    for sec, kv in TUBE_INI.items():
        for k, v in kv.items():
            cfg.set(sec, k, v)
    cfg.set("grid", "nxmax", nx)
    cfg.set("grid", "nymax", ny)
    if ny > 1:
        cfg.set("grid", "domain_size_y", repr(0.01 * ny / 128.0))
    if tables is None:
        tables = M.build_tables(mechanism("shock_tube_9sp"), 7173.0, 200.0, 20000.0, 1.0)
    return CS.Case(cfg, tables)


def config1_case(nx: int = 2400, cfl: float = 0.5, tables: M.Tables = None):
    """The 1-D reactive shock tube on nx cells over 0.12 m with a CFL-driven step
    (the reference's example, examples/reactive_shock_tube, runs 400 cells at a
    fixed dt of 2e-8 s): reflecting wall at x = 0, extrapolation at x = 0.12 m,
    H2:O2:Ar = 2:1:7 with the example's 9-species, 18-reaction mechanism, the
    example's initial step at 0.06 m (left rho = 0.072, p = 7173 Pa, u = 0; right
    rho = 0.18075, p = 35594 Pa, u = -487.34 m/s), WENO5 on every face,
    Strang + ROK4."""
    c = tube_case(nx, tables=tables)
    c.cfl = cfl
    return c


def flame_case(nx: int, phi: float = 0.6, Tu: float = 298.0, tables: M.Tables = None, L: float = 0.03,
               delta: float = 3e-4, mech_name: str = "flame_11sp"):
    """A 1-D laminar premixed H2/air flame on nx cells of an L-long domain: the
    settings of examples/laminar_premix_flame (11 species by default, or the
    9-species H2/air mechanism with mech_name="h2air_9sp"; inflow at xmin,
    extrapolation at xmax, WENO5-Z everywhere with KEEP(2), "simpler" splitting
    with ROK4, fixed dt 1e-8 s).  The reference reads its profile from
    premix.dat; here a synthetic flame of the same shape stands in: T, Y blend
    between the unburnt mixture (equivalence ratio phi, Tu, 1 atm) and its
    complete-combustion products at the adiabatic temperature through a tanh of
    thickness delta at L/2, with constant mass flux rho u."""
    mech = mechanism(mech_name)
    if tables is None:
        tables = M.build_tables(mech, 101325.0, 200.0, 5500.0, 1.0)
    ns = mech.ns
    iH2, iO2, iH2O, iN2 = mech.index("H2"), mech.index("O2"), mech.index("H2O"), mech.index("N2")
    mw = np.array([s.mw for s in mech.species])
    X = np.zeros(ns)
    X[iH2], X[iO2], X[iN2] = 2.0 * phi, 1.0, 3.76
    Yu = X * mw / np.dot(X, mw)
    # complete combustion 2 H2 + O2 -> 2 H2O (per unit mass of mixture)
    nH2, nO2 = Yu[iH2] / mw[iH2], Yu[iO2] / mw[iO2]
    burn = min(nH2, 2.0 * nO2)
    Yb = Yu.copy()
    Yb[iH2] -= burn * mw[iH2]
    Yb[iO2] -= 0.5 * burn * mw[iO2]
    Yb[iH2O] += burn * mw[iH2O]
    Yb = np.maximum(Yb, 0.0)
    Yb /= Yb.sum()
    hu = M.mixture_h(tables, Tu, Yu)
    Tb = 2000.0
    for _ in range(50):           # adiabatic T of the products (constant p): h(Tb, Yb) = h(Tu, Yu)
        f = M.mixture_h(tables, Tb, Yb) - hu
        Tb -= f / M.mixture_cp(tables, Tb, Yb)
        if abs(f) < 1e-9 * abs(hu) + 1e-6:
            break
    p0 = 101325.0
    rho_u = p0 / (np.dot(tables.rgas, Yu) * Tu)
    su = 0.9139672490375892        # inflow speed of the reference's flame case
    cfg = CS.default_ini(nx, 1, 1, L=(L, 1.0, 1.0), bc=(1, 2, 0, 0, 0, 0), t0=Tu, p0=p0, Y=Yu, ns=ns,
                         chemistry=2, rosenbrock_version=2, splitting=1, weno_version=1, sensor_threshold=-0.2,
                         sensor_type=0, nkeep=2, ep_order=6, flux_splitting=0, cfl=-1e-8, flow_init=100)
    cfg.set("ref_state", "u0", repr(su))
    c = CS.Case(cfg, tables)
    ng = c.ng
    x = c.x[ng:ng + nx]
    s = 0.5 * (1.0 + np.tanh((x - 0.5 * L) / delta))
    T = (1.0 - s) * Tu + s * Tb
    Y = (1.0 - s)[None, :] * Yu[:, None] + s[None, :] * Yb[:, None]
    rho = p0 / (np.einsum("k,kx->x", tables.rgas, Y) * T)
    u = rho_u * su / rho
    sh = (1, 1, nx)
    c.set_interior(rho.reshape(sh), u.reshape(sh), np.zeros(sh), np.zeros(sh), T.reshape(sh),
                   Y.reshape((ns,) + sh))
    c.flame = dict(phi=phi, Tu=Tu, Tb=Tb, Yu=Yu, Yb=Yb)
    return c


# The laminar premixed flame's inputs (examples/laminar_premix_flame/multideal.ini):
# 11-species, 21-reaction H2/O2 mechanism with Ar/He/N2, 2000 cells over 3 cm,
# inflow (bc 1) at xmin and extrapolation at xmax, WENO5-Z on every face
# (threshold -0.2) with KEEP(2), "simpler" splitting with ROK4, fixed dt 1e-8 s;
# the initial profile is premix.dat (flow_init 10).
FLAME_INI = {
    "ref_state": {"t0": "298.", "p0": "101325.0", "u0": "0.9139672490375892",
                  "init_Y_01": "0.0173109321627845", "init_Y_02": "0.", "init_Y_03": "0.2289662728773070",
                  "init_Y_04": "0.", "init_Y_05": "0.", "init_Y_06": "0.", "init_Y_07": "0.", "init_Y_08": "0.",
                  "init_Y_09": "0.", "init_Y_10": "0.", "init_Y_11": "0.7537227949599082"},
    "grid": {"domain_size_x": "0.03", "domain_size_y": "1.", "domain_size_z": "1.", "nxmax": "2000", "nymax": "1",
             "nzmax": "1", "ng": "3", "metrics_order": "6", "grid_type": "2"},
    "bc": {"xmin": "1", "xmax": "2", "ymin": "0", "ymax": "0", "zmin": "0", "zmax": "0", "xmin_nr": "0",
           "xmax_nr": "0", "ymin_nr": "0", "ymax_nr": "0", "zmin_nr": "0", "zmax_nr": "0"},
    "controls": {"cfl": "-1E-8", "iter_dt_recompute": "1", "num_iter": "100000"},
    "numerics": {"ep_order": "6", "nkeep": "2", "visc_order": "6", "conservative_viscous": "1", "weno_scheme": "3",
                 "weno_version": "1", "flux_splitting": "0", "sensor_threshold": "-0.2", "sensor_type": "0",
                 "rk_type": "1", "ros_dttry": "1.e-9", "ros_eps": "1.e-8", "ros_maxsteps": "10000",
                 "ros_maxtry": "40", "operator_splitting": "1", "rosenbrock_version": "2"},
    "flow": {"flow_init": "10"},
    "fluid": {"use_cantera": "1", "enable_chemistry": "2", "t_min_tab": "200.", "t_max_tab": "20000.",
              "dt_tab": "1."},
}


def premix_profile():
    """The reference flame's initial profile (premix.dat of examples/laminar_premix_flame):
    x, u, T (2000 cells) and Y (11, 2000)."""
    d = np.load(os.path.join(DATA, "premix_flame_11sp.npz"))
    return d["x"], d["u"], d["T"], d["Y"]


def premix_flame_case(nx: int = 2000, tables: M.Tables = None, visc_scale: float = 1.0, lam_scale: float = 1.0,
                      diff_scale: float = 1.0):
    """The reference's laminar premixed flame run (examples/laminar_premix_flame):
    its multideal.ini and its premix.dat profile (the first nx cells of it when
    nx < 2000, with the domain shortened to keep the spacing).  visc_scale,
    lam_scale and diff_scale multiply the species viscosity, conductivity and
    binary-diffusion tables (sensitivity knobs for the transport tables, which
    come from the project's kinetic-theory generator instead of Cantera)."""
    cfg = CS.Config()
    for sec, kv in FLAME_INI.items():
        for k, v in kv.items():
            cfg.set(sec, k, v)
    if nx != 2000:
        cfg.set("grid", "nxmax", nx)
        cfg.set("grid", "domain_size_x", repr(0.03 * (nx - 1) / 1999.0))
    if tables is None:
        tables = M.build_tables(mechanism("flame_11sp"), 101325.0, 200.0, 20000.0, 1.0)
    if visc_scale != 1.0 or lam_scale != 1.0 or diff_scale != 1.0:
        import copy
        tables = copy.copy(tables)
        tables.visc = tables.visc * visc_scale
        tables.lam = tables.lam * lam_scale
        tables.diffbin = tables.diffbin * diff_scale
    c = CS.Case(cfg, tables)
    _, u, T, Y = premix_profile()
    c.init_premix(u, T, Y)
    return c


def stiff_mechanism_tables(seed: int = 0):
    mech = M.synthetic_mechanism(53, 325, seed)
    return mech, M.build_tables(mech, 101325.0, 200.0, 5500.0, 1.0)


def stiff_case(n: int, seed: int = 0, tables: M.Tables = None, dt: float = 1e-9, rosenbrock_version: int = 1):
    """The stiff-mechanism scaling workload on an n^3 periodic box (side
    2 pi mm n/128): 53 species / 325 reactions (stx.mech.synthetic_mechanism),
    p = 1 atm, Y ~ Dirichlet(0.5) per cell and T on a smooth random field in
    1200..2000 K (both seeded), at rest; WENO5-Z / KEEP(2) hybrid (threshold 0.1),
    Strang splitting with the full-Jacobian Rosenbrock (rosenbrock_version 1: the
    dense (ns+4)^2 Jacobian; the 4-vector Krylov basis of ROK4 cannot follow 53
    stiff modes and caps its step count), fixed dt."""
    if tables is None:
        _, tables = stiff_mechanism_tables(seed)
    ns = tables.ns
    rng = np.random.default_rng(seed + 1)
    L = 2.0 * math.pi * 1e-3 * n / 128.0
    cfg = CS.default_ini(n, n, n, L=(L, L, L), bc=(0,) * 6, t0=1600.0, p0=101325.0, Y=np.full(ns, 1.0 / ns), ns=ns,
                         chemistry=2, rosenbrock_version=rosenbrock_version, splitting=2, weno_version=1,
                         sensor_threshold=0.1, sensor_type=1, nkeep=2, ep_order=6, flux_splitting=0, cfl=-dt,
                         flow_init=100)
    c = CS.Case(cfg, tables)
    # smooth T: a few seeded Fourier modes, scaled to [-1, 1]
    x = (np.arange(n) + 0.5) / n * 2.0 * math.pi
    X, Yg, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.zeros((n, n, n))
    for _ in range(6):
        k = rng.integers(1, 4, size=3)
        ph = rng.uniform(0, 2 * math.pi, size=3)
        f += np.sin(k[0] * X + ph[0]) * np.sin(k[1] * Yg + ph[1]) * np.sin(k[2] * Z + ph[2])
    f = f / np.abs(f).max()
    T = (1600.0 + 400.0 * f).transpose(2, 1, 0)            # (nz, ny, nx)
    Yc = rng.dirichlet(np.full(ns, 0.5), size=(n, n, n))   # (nz, ny, nx, ns)
    Yc = np.moveaxis(Yc, -1, 0)
    rho = 101325.0 / (np.einsum("k,kzyx->zyx", tables.rgas, Yc) * T)
    zero = np.zeros_like(T)
    c.set_interior(rho, zero, zero, zero, T, Yc)
    return c


def shock_tube_case(nx: int, cfg_keys: dict, mech_name="shock_tube_9sp"):
    cfg = CS.Config()
    for sec, kv in cfg_keys.items():
        for k, v in kv.items():
            cfg.set(sec, k, v)
    cfg.set("grid", "nxmax", nx)
    tb = M.build_tables(mechanism(mech_name), cfg.get("ref_state", "p0"), cfg.get("fluid", "t_min_tab"),
                        cfg.get("fluid", "t_max_tab"), cfg.get("fluid", "dt_tab"))
    return CS.Case(cfg, tb)
