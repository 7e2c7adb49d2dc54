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
            out.append(np.fft.irfftn(a - kc * dot, s=(n, n, n)))
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


def shock_tube_case(nx: int, cfg_keys: dict, mech_name="shock_tube_9sp"):
    cfg = CS.Config()
    for sec, kv in cfg_keys.items():
        for k, v in kv.items():
            cfg.set(sec, k, v)
    cfg.set("grid", "nxmax", nx)
    tb = M.build_tables(mechanism(mech_name), cfg.get("ref_state", "p0"), cfg.get("fluid", "t_min_tab"),
                        cfg.get("fluid", "t_max_tab"), cfg.get("fluid", "dt_tab"))
    return CS.Case(cfg, tb)
