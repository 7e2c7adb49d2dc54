"""Host logic of the served mix and of the batched-reactor workload, no GPU:
the seeded request stream (Poisson arrivals; 60 % 0-D reactors, 30 % 1-D
flames with nx ~ U{512..4096}, phi ~ U(0.5, 1.5), Tu ~ U(300, 800) K, 10 % 2-D
shock tubes of 512 x 128 cells) and the reactor sample (T0 ~ U(900, 1500) K,
p ~ logU(1, 40) atm, phi ~ U(0.3, 3), H2/air with O2:N2 = 1:3.76)."""
import numpy as np

import helpers as H  # noqa: F401  (puts the package on sys.path)
from stx import configs
from stx.reactors import sample_h2air
from stx.requests import mixed_requests

MECH = configs.mechanism("h2air_9sp")


def test_request_stream_is_seeded_poisson_with_the_stated_mix():
    n, rate = 10000, 10.0
    reqs = mixed_requests(n, rate, 7, MECH)
    again = mixed_requests(n, rate, 7, MECH)
    assert [(r.kind, r.arrival, r.steps) for r in reqs] == [(r.kind, r.arrival, r.steps) for r in again]
    assert [r.rid for r in reqs] == list(range(n))
    t = np.array([r.arrival for r in reqs])
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert np.all(gaps > 0.0)
    # exponential gaps: mean 1/rate (standard error 1 % at n = 10^4), coefficient of variation 1
    assert abs(gaps.mean() * rate - 1.0) < 0.03
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05
    kinds = np.array([r.kind for r in reqs])
    for kind, frac in (("reactor", 0.6), ("flame1d", 0.3), ("tube2d", 0.1)):
        assert abs(np.mean(kinds == kind) - frac) < 0.02, kind
    other = mixed_requests(n, rate, 8, MECH)
    assert [r.arrival for r in other] != [r.arrival for r in reqs]


def test_request_parameters_stay_in_their_ranges():
    reqs = mixed_requests(3000, 5.0, 11, MECH, flame_steps=20, tube_steps=10)
    flames = [r for r in reqs if r.kind == "flame1d"]
    tubes = [r for r in reqs if r.kind == "tube2d"]
    reactors = [r for r in reqs if r.kind == "reactor"]
    nx = np.array([r.params["nx"] for r in flames])
    assert nx.min() >= 512 and nx.max() <= 4096 and len(np.unique(nx)) > 100
    assert all(0.5 <= r.params["phi"] <= 1.5 and 300.0 <= r.params["Tu"] <= 800.0 for r in flames)
    assert all(r.steps == 20 for r in flames)
    assert all(r.params == {"nx": 512, "ny": 128} and r.steps == 10 for r in tubes)
    for r in reactors:
        assert 900.0 <= r.params["T0"] <= 1500.0
        assert 101325.0 <= r.params["p0"] <= 40 * 101325.0
        assert r.params["Y0"].shape == (MECH.ns,)
        assert abs(r.params["Y0"].sum() - 1.0) < 1e-12


def test_reactor_sample_is_h2_air_at_the_stated_ranges():
    n = 4000
    T0, p0, Y0 = sample_h2air(n, 3, MECH)
    assert T0.shape == (n,) and p0.shape == (n,) and Y0.shape == (MECH.ns, n)
    assert T0.min() >= 900.0 and T0.max() <= 1500.0
    patm = p0 / 101325.0
    assert patm.min() >= 1.0 and patm.max() <= 40.0
    # log-uniform pressure: log p is uniform on [0, ln 40] (mean ln 40 / 2)
    assert abs(np.log(patm).mean() - 0.5 * np.log(40.0)) < 0.05
    assert np.all(Y0 >= 0.0) and np.max(np.abs(Y0.sum(axis=0) - 1.0)) < 1e-12
    mw = np.array([s.mw for s in MECH.species])
    X = Y0 / mw[:, None]
    X = X / X.sum(axis=0)
    iH2, iO2, iN2 = MECH.index("H2"), MECH.index("O2"), MECH.index("N2")
    np.testing.assert_allclose(X[iN2] / X[iO2], 3.76, rtol=1e-12)
    phi = X[iH2] / (2.0 * X[iO2])
    assert phi.min() >= 0.3 and phi.max() <= 3.0
    others = [k for k in range(MECH.ns) if k not in (iH2, iO2, iN2)]
    assert np.all(Y0[others] == 0.0)
    again = sample_h2air(n, 3, MECH)
    assert all(np.array_equal(a, b) for a, b in zip((T0, p0, Y0), again))
