"""The workloads' inputs, built on the host, against their descriptions:
  * the turbulence box (numpy and torch on the CPU): a random-phase solenoidal
    velocity with E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4, scaled to u_rms = 0.3 c0
    of the mean state (9-species H2/air, phi = 0.7, T = 1000 K, p = 1 atm), the
    ghost points holding the mean state at rest;
  * the 53-species / 325-reaction stiff mechanism and its box;
  * the 2400-cell reactive shock tube's initial state."""
import math

import numpy as np
import pytest
import torch

import helpers as H  # noqa: F401  (puts the package on sys.path)
from stx import configs
from stx import mech as M

N = 32


def _spectral(u, v, w):
    n = u.shape[0]
    U, V, W = (np.fft.rfftn(a) for a in (u, v, w))
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    kr = np.fft.rfftfreq(n, d=1.0 / n)
    kx, ky, kz = kr[None, None, :], k1[None, :, None], k1[:, None, None]
    return U, V, W, kx, ky, kz


@pytest.mark.parametrize("xp", ["numpy", "torch"])
def test_velocity_is_solenoidal_with_the_stated_spectrum(xp):
    lib = np if xp == "numpy" else torch
    u, v, w = configs.turbulence_velocity(N, 5, 4.0, xp=lib, device=None if xp == "numpy" else "cpu")
    if xp == "torch":
        u, v, w = u.numpy(), v.numpy(), w.numpy()
    assert u.shape == (N, N, N) and u.dtype == np.float64
    U, V, W, kx, ky, kz = _spectral(u, v, w)
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    # the divergence k . u_hat vanishes to rounding away from the Nyquist
    # planes (where a real field's +-n/2 partner modes share one coefficient)
    inner = (np.abs(kx) < N / 2) & (np.abs(ky) < N / 2) & (np.abs(kz) < N / 2)
    amp = np.sqrt(np.abs(U) ** 2 + np.abs(V) ** 2 + np.abs(W) ** 2)
    div = np.abs(kx * U + ky * V + kz * W)
    assert div[inner].max() < 1e-12 * (kk * amp).max()
    # zero mean; the shell spectrum follows k^4 exp(-2 (k/4)^2) within the
    # scatter of a few hundred random modes per shell, and peaks at k0
    assert max(abs(float(a.mean())) for a in (u, v, w)) < 1e-15
    e = amp ** 2 * np.where(kx > 0, 2.0, 1.0)          # the rfft half-space counts its mirror once
    shell = np.rint(kk).astype(int)
    E = np.bincount(shell.ravel(), e.ravel())
    ks = np.arange(3, 12)
    model = ks ** 4.0 * np.exp(-2.0 * (ks / 4.0) ** 2)
    r = E[ks] / model
    r = r / r.mean()
    assert r.min() > 0.6 and r.max() < 1.5, r
    assert 3 <= int(np.argmax(E[1:N // 2])) + 1 <= 5


def test_turbulence_state_has_the_stated_mean_state_and_rms():
    case = configs.turbulence_case(N)
    W, WA = configs.turbulence_fields(case, 9)
    p, tb, Y, ns, ng = case.turb, case.tb, case.turb_Y, case.ns, case.ng
    assert (p["T0"], p["p0"], p["phi"], p["mach_rms"], p["k0"]) == (1000.0, 101325.0, 0.7, 0.3, 4.0)
    np.testing.assert_allclose(Y, configs.h2air_Y(0.7, configs.mechanism("h2air_9sp")), rtol=0, atol=1e-15)
    rm = float(np.dot(tb.rgas, Y))
    rho = p["p0"] / (rm * p["T0"])
    cp = M.mixture_cp(tb, p["T0"], Y)
    c0 = math.sqrt(cp / (cp - rm) * rm * p["T0"])
    e0 = M.mixture_e(tb, p["T0"], Y)
    assert W.shape == (case.nv, case.nzg, case.nyg, case.nxg)
    interior = (slice(ng, ng + N),) * 3
    r = W[:ns].sum(axis=0)
    np.testing.assert_allclose(r, rho, rtol=1e-14)
    vel = [W[(ns + m,) + interior] / rho for m in range(3)]
    rms = math.sqrt(sum(float((a * a).mean()) for a in vel) / 3.0)
    assert abs(rms / (0.3 * c0) - 1.0) < 1e-12
    ke = 0.5 * sum(a * a for a in vel)
    np.testing.assert_allclose(W[(ns + 3,) + interior], rho * (e0 + ke), rtol=1e-13)
    # ghosts: the mean state at rest
    ghost = np.ones((case.nzg, case.nyg, case.nxg), bool)
    ghost[interior] = False
    for m in range(3):
        assert np.all(W[ns + m][ghost] == 0.0)
    np.testing.assert_allclose(W[ns + 3][ghost], rho * e0, rtol=1e-14)
    assert np.all(WA[case.J("T")] == p["T0"])
    # a same-resolution sample: the grid spacing is that of the 256^3 box
    for xg in case.xg:
        np.testing.assert_allclose(np.diff(xg), 2.0 * math.pi * p["ell"] / 256, rtol=1e-12)


def test_stiff_mechanism_has_the_stated_distributions():
    """The 53-species / 325-reaction workload: A ~ logU(1e8, 1e16) (cm, mol
    units), b ~ U(-1.5, 2), Ea ~ U(0, 50) kcal/mol, about 20 % three-body
    reactions with efficiencies U(0.5, 5); every reaction reversible and
    bimolecular between four distinct species of one molecular weight; NASA-7
    coefficients within 5 % of N2's."""
    mech = M.synthetic_mechanism(53, 325, 0)
    assert len(mech.species) == 53 and len(mech.reactions) == 325
    mw = {s.mw for s in mech.species}
    assert len(mw) == 1
    n2 = [[3.298677, 0.0014082404, -3.963222e-06, 5.641515e-09, -2.444854e-12, -1020.8999, 3.950372],
          [2.92664, 0.0014879768, -5.68476e-07, 1.0097038e-10, -6.753351e-15, -922.7977, 5.980528]]
    for s in mech.species:
        r = np.array(s.coeffs) / np.array(n2)
        assert r.min() >= 0.95 and r.max() <= 1.05
    cal = 4.184e6
    three = 0
    for r in mech.reactions:
        assert r.reversible
        names = list(r.reactants) + list(r.products)
        assert len(set(names)) == 4 and all(v == 1.0 for v in list(r.reactants.values()) + list(r.products.values()))
        A, b, Ea = r.rate
        if r.efficiencies is not None:
            three += 1
            A_cgs = A / (1e-6 / 1e-3) ** 2
            effs = np.array(list(r.efficiencies.values()))
            assert len(effs) == 53 and effs.min() >= 0.5 and effs.max() <= 5.0
        else:
            A_cgs = A / (1e-6 / 1e-3)
        assert 8.0 <= math.log10(A_cgs) <= 16.0
        assert -1.5 <= b <= 2.0 and 0.0 <= Ea / cal <= 50.0
    assert 0.14 < three / 325 < 0.26
    assert M.synthetic_mechanism(53, 325, 0).reactions[17].rate == mech.reactions[17].rate


def test_stiff_case_state():
    """The 53-species box: p = 1 atm at rest, T a smooth seeded field spanning
    1200..2000 K, Y_k ~ Dirichlet(0.5) per cell."""
    n = 8
    mech, tables = configs.stiff_mechanism_tables(0)
    case = configs.stiff_case(n, tables=tables)
    ns, ng = case.ns, case.ng
    assert ns == 53 and case.nv == 57
    sl = (slice(ng, ng + n),) * 3
    w = case.w
    rho = w[(slice(0, ns),) + sl].sum(axis=0)
    Y = w[(slice(0, ns),) + sl] / rho[None]
    assert Y.min() >= 0.0 and np.max(np.abs(Y.sum(axis=0) - 1.0)) < 1e-13
    # Dirichlet(0.5) over 53 species: E[Y_k] = 1/53, Var = (1/53)(52/53)/(53*0.5 + 1)
    assert abs(Y.mean() - 1.0 / 53) < 1e-12
    assert abs(Y.var() / ((1.0 / 53) * (52.0 / 53) / 27.5) - 1.0) < 0.1
    for m in range(3):
        assert np.all(w[(ns + m,) + sl] == 0.0)
    T = case.w_aux[(case.J("T"),) + sl]
    assert T.min() >= 1200.0 - 1e-9 and T.max() <= 2000.0 + 1e-9 and T.max() - T.min() > 600.0
    rm = np.einsum("k,kzyx->zyx", tables.rgas, Y)
    np.testing.assert_allclose(rho * rm * T, 101325.0, rtol=1e-12)


def _T_from_e(tb, e, Y, lo=200.0, hi=5000.0):
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if M.mixture_e(tb, mid, Y) < e:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def test_config1_shock_tube_initial_state():
    """The 2400-cell reactive shock tube: H2:O2:Ar = 2:1:7 by moles over 0.12 m,
    left state rho = 0.072 kg/m^3, p = 7173 Pa at rest, right state (x >= 0.06 m)
    rho = 0.18075 kg/m^3, p = 35594 Pa, u = -487.34 m/s."""
    c = configs.config1_case(2400)
    ns, ng, nx = c.ns, c.ng, c.nx
    assert nx == 2400 and c.cfl == 0.5
    x = np.asarray(c.x)[ng:ng + nx]
    assert x[0] == 0.0 and abs(x[-1] - 0.12) < 1e-15
    w = c.w[:, ng, ng, ng:ng + nx]
    rho = w[:ns].sum(axis=0)
    Y = w[:ns] / rho[None]
    mech = configs.mechanism("shock_tube_9sp")
    mw = np.array([s.mw for s in mech.species])
    X = Y / mw[:, None]
    X = X / X.sum(axis=0)
    # the example's mass fractions (multideal.ini init_Y_*), which are 2:1:7 by
    # moles to within 0.7 %
    for k in range(ns):
        np.testing.assert_allclose(Y[k], float(configs.TUBE_INI["ref_state"]["init_Y_%02d" % (k + 1)]),
                                   rtol=1e-13, atol=1e-16)
    for name, frac in (("H2", 0.2), ("O2", 0.1), ("AR", 0.7)):
        k = [s.name.upper() for s in mech.species].index(name)
        np.testing.assert_allclose(X[k], frac, rtol=7e-3)
    right = x >= 0.06
    assert right.sum() == nx // 2
    u = w[ns] / rho
    tb = c.tb
    for sel, r0, u0, p0 in ((~right, 0.072, 0.0, 7173.0), (right, 0.18075, -487.34, 35594.0)):
        i = np.flatnonzero(sel)[[0, -1]]
        np.testing.assert_allclose(rho[i], r0, rtol=1e-14)
        np.testing.assert_allclose(u[i], u0, rtol=1e-14, atol=1e-14)
        for j in i:
            e = w[ns + 3, j] / rho[j] - 0.5 * u[j] ** 2
            T = _T_from_e(tb, e, Y[:, j])
            assert abs(rho[j] * float(np.dot(tb.rgas, Y[:, j])) * T / p0 - 1.0) < 1e-9
