"""tau_int estimator against series with known integrated autocorrelation time."""
import numpy as np
import pytest

from cuda_pspin_b200 import tau as T


def ar1(phi, n, chains, seed):
    rng = np.random.default_rng(seed)
    e = rng.normal(size=(chains, n))
    x = np.empty_like(e)
    x[:, 0] = e[:, 0] / np.sqrt(1 - phi * phi)
    for t in range(1, n):
        x[:, t] = phi * x[:, t - 1] + e[:, t]
    return x


@pytest.mark.parametrize("phi", [0.0, 0.5, 0.9, 0.97])
def test_ar1_tau_int(phi):
    """AR(1): rho(t) = phi^t, tau_int = (1 + phi) / (2 (1 - phi))."""
    x = ar1(phi, 20000, 16, seed=int(phi * 100))
    r = T.tau_int(x)
    exact = (1 + phi) / (2 * (1 - phi))
    assert abs(r.tau - exact) < 4 * r.err + 0.02, (r, exact)
    assert r.err < 0.1 * exact + 0.02


def test_window_rule():
    r = T.tau_int(ar1(0.9, 20000, 8, seed=3))
    assert r.window >= 5 * r.tau - 1 and r.window < 5 * r.tau + 5


def test_single_chain_and_constant():
    r = T.tau_int(ar1(0.5, 50000, 1, seed=4)[0])
    assert abs(r.tau - 1.5) < 0.2
    c = T.tau_int(np.ones(100))
    assert c.tau == 0.5


def test_exp_crossing_ar1():
    """rho(t) = phi^t crosses 1/e at t = -1/ln(phi) (interpolated)."""
    phi = 0.9
    x = ar1(phi, 400000, 1, seed=5)[0]
    assert abs(T.tau_exp_crossing(x) - (-1.0 / np.log(phi))) < 0.5


def test_autocovariance_matches_direct():
    x = ar1(0.7, 300, 3, seed=6)
    c = T.autocovariance(x)
    y = x - x.mean(axis=1, keepdims=True)
    for t in (0, 1, 5, 40):
        direct = np.mean([np.dot(y[k, :300 - t], y[k, t:]) / (300 - t) for k in range(3)])
        assert abs(c[t] - direct) < 1e-12
