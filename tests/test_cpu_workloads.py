"""The synthetic turbulence workload, built on the host (numpy and torch on the
CPU), against its description: a random-phase solenoidal velocity with
E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4, scaled to u_rms = 0.3 c0 of the mean
state (9-species H2/air, phi = 0.7, T = 1000 K, p = 1 atm), on a box whose
ghost points hold the mean state at rest."""
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
