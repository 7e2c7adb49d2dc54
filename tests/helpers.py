"""Shared test helpers: case builders from the committed fixtures, oracle access,
and comparison utilities."""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "prop-streams2_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

from stx import case as CS  # noqa: E402
from stx import mech as M  # noqa: E402

GOLDEN = os.path.join(HERE, "golden")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as fh:
        return json.load(fh)


def mechanism(name: str) -> M.Mechanism:
    return M.mechanism_from_dict(golden(f"mech_{name}.json"))


_TABLE_CACHE = {}


def tables(name: str, p0: float, tmin=200.0, tmax=5500.0, dtab=1.0) -> M.Tables:
    key = (name, p0, tmin, tmax, dtab)
    if key not in _TABLE_CACHE:
        _TABLE_CACHE[key] = M.build_tables(mechanism(name), p0, tmin, tmax, dtab)
    return _TABLE_CACHE[key]


def h2air_Y(phi: float, mech: M.Mechanism) -> np.ndarray:
    """Mass fractions of an H2/air (O2:N2 = 1:3.76) premixture at equivalence ratio phi."""
    X = np.zeros(mech.ns)
    X[mech.index("H2")] = 2.0 * phi
    X[mech.index("O2")] = 1.0
    X[mech.index("N2")] = 3.76
    X /= X.sum()
    mw = np.array([s.mw for s in mech.species])
    Y = X * mw
    return Y / Y.sum()


def synthetic_case(n=(16, 12, 10), mech="h2air_9sp", seed=0, bc=(0, 0, 0, 0, 0, 0), amp_u=60.0, amp_T=150.0,
                   T0=1100.0, p0=101325.0, phi=0.7, L=(0.01, 0.008, 0.006), **kw):
    """A smooth random field on a small grid for kernel parity tests."""
    mm = mechanism(mech)
    Y0 = h2air_Y(phi, mm) if "N2" in mm.names else None
    if Y0 is None:
        Y0 = np.zeros(mm.ns)
        Y0[mm.index("H2")] = 0.0127
        Y0[mm.index("O2")] = 0.1014
        Y0[mm.index("Ar")] = 1.0 - Y0.sum()
    cfg = CS.default_ini(n[0], n[1], n[2], L=L, bc=bc, t0=T0, p0=p0, Y=Y0, ns=mm.ns, **kw)
    tb = tables(mech, p0)
    case = CS.Case(cfg, tb)
    rng = np.random.default_rng(seed)
    nz, ny, nx = n[2], n[1], n[0]
    z, y, x = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")

    def smooth(a):
        f = np.zeros_like(x)
        for _ in range(3):
            kx, ky, kz = rng.integers(1, 3, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            f += rng.uniform(-1, 1) * np.sin(2 * np.pi * kx * x + ph[0]) * np.cos(2 * np.pi * ky * y + ph[1]) * \
                np.sin(2 * np.pi * kz * z + ph[2])
        return a * f / 3.0

    T = T0 + smooth(amp_T)
    u, v, w = smooth(amp_u), smooth(amp_u), smooth(amp_u)
    Y = np.empty((mm.ns,) + x.shape)
    for k in range(mm.ns):
        Y[k] = Y0[k] * (1.0 + 0.2 * smooth(1.0)) + (1e-4 if Y0[k] == 0 else 0.0) * (1.0 + smooth(0.5))
    Y /= Y.sum(axis=0)
    rm = np.tensordot(tb.rgas, Y, axes=1)
    p = p0 * (1.0 + smooth(0.05))
    rho = p / (rm * T)
    case.set_interior(rho, u, v, w, T, Y)
    return case


def batch_case(nx=1, ny=1, nz=1):
    """The reference's 0-D batch reactor (examples/batch_reactor) on an nx x ny x nz periodic box."""
    g = golden("batch_reactor_keromnes.json")
    cfg = CS.Config()
    for sec, kv in g["ini"].items():
        for k, v in kv.items():
            cfg.set(sec, k, v)
    for a, n in zip("xyz", (nx, ny, nz)):
        cfg.set("grid", f"n{a}max", n)
    tb = tables("keromnes_14sp", cfg.get("ref_state", "p0"), cfg.get("fluid", "t_min_tab"),
                cfg.get("fluid", "t_max_tab"), cfg.get("fluid", "dt_tab"))
    return CS.Case(cfg, tb), g


def shock_tube_case(nx=400, mech="shock_tube_9sp"):
    """The reference's reactive shock tube (examples/reactive_shock_tube) inputs."""
    ini = golden("shock_tube_ini.json")
    cfg = CS.Config()
    for sec, kv in ini.items():
        for k, v in kv.items():
            cfg.set(sec, k, v)
    cfg.set("grid", "nxmax", nx)
    p0 = cfg.get("ref_state", "p0")
    tb = tables(mech, p0, cfg.get("fluid", "t_min_tab"), cfg.get("fluid", "t_max_tab"), cfg.get("fluid", "dt_tab"))
    return CS.Case(cfg, tb)


def assert_close(gpu, ref, rtol, name="", floor=None):
    """|gpu - ref| <= rtol * max(|ref|, floor) elementwise, floor defaulting to rtol-scaled field max."""
    gpu = np.asarray(gpu)
    ref = np.asarray(ref)
    assert gpu.shape == ref.shape, (name, gpu.shape, ref.shape)
    scale = np.max(np.abs(ref)) if floor is None else floor
    tol = rtol * np.maximum(np.abs(ref), scale * 1e-3 if floor is None else floor)
    err = np.abs(gpu - ref)
    bad = err > tol
    if np.any(bad) or not np.all(np.isfinite(gpu) == np.isfinite(ref)):
        idx = np.unravel_index(np.argmax(err - tol), err.shape)
        raise AssertionError(f"{name}: max err {err.max():.3e} at {idx}: gpu={gpu[idx]!r} ref={ref[idx]!r} "
                             f"({bad.sum()} of {bad.size} outside rtol={rtol})")


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
