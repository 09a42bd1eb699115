"""Integrated autocorrelation time of Monte Carlo series.

tau_int with Sokal's automatic windowing (Madras & Sokal, J. Stat. Phys. 50,
109 (1988); Sokal, "Monte Carlo methods in statistical mechanics", 1996):

    rho(t)     = C(t) / C(0),  C(t) = <(x_s - m)(x_{s+t} - m)>
    tau(W)     = 1/2 + sum_{t=1..W} rho(t)
    W          = the smallest window with W >= c * tau(W)   (c = 5 here)
    var(tau)  ~= 2 (2W + 1) / n * tau^2

so that the variance of a time average of n correlated samples is
2 tau_int var(x) / n and a chain delivers n / (2 tau_int) independent
samples.  Several independent chains (disorder samples, replicas) are
combined by averaging their autocovariance functions, each chain about its
own mean.

Also the reference's decorrelation time: the lag at which the normalised
autocorrelation of the second half of the series first drops below 1/e,
linearly interpolated (analysis_pt.cpp:2694-2770).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Tau:
    tau: float          # tau_int in units of the series spacing
    window: int         # Sokal window W
    err: float          # statistical error of tau (Madras-Sokal)
    n: int              # length of each chain
    chains: int


def autocovariance(x) -> np.ndarray:
    """Mean over chains of C(t), t = 0..n-1; x is [n] or [chains, n]."""
    x = np.atleast_2d(np.asarray(x, np.float64))
    n = x.shape[1]
    y = x - x.mean(axis=1, keepdims=True)
    m = 1 << int(np.ceil(np.log2(2 * n)))
    f = np.fft.rfft(y, m, axis=1)
    c = np.fft.irfft(f * np.conj(f), m, axis=1)[:, :n]
    c /= (n - np.arange(n))            # unbiased at each lag
    return c.mean(axis=0)


def tau_int(x, c: float = 5.0) -> Tau:
    """Sokal automatic-window estimate over a series [n] or chains [chains, n]."""
    x = np.atleast_2d(np.asarray(x, np.float64))
    chains, n = x.shape
    if n < 4:
        raise ValueError("series too short")
    cov = autocovariance(x)
    if cov[0] <= 0.0:
        return Tau(0.5, 0, 0.0, n, chains)
    rho = cov / cov[0]
    tau = 0.5
    W = n - 1
    for t in range(1, n):
        tau += rho[t]
        if t >= c * tau:
            W = t
            break
    err = tau * np.sqrt(2.0 * (2 * W + 1) / (n * chains))
    return Tau(float(tau), int(W), float(err), n, chains)


def tau_exp_crossing(x) -> float:
    """The reference's tau_E: 1/e crossing of rho over the second half of one
    series (replica-averaged by the caller), linearly interpolated; n/2 - 1
    when it never crosses."""
    x = np.asarray(x, np.float64)
    M = len(x)
    e = x[M // 2:]
    n = len(e)
    if n < 4:
        return 0.0
    m = e.mean()
    var = (e * e).mean() - m * m
    if var <= 0.0:
        return 0.0
    d = e - m
    inv_e = np.exp(-1.0)
    prev_rho = 1.0
    for lag in range(1, n // 2):
        rho = float(np.dot(d[:n - lag], d[lag:]) / (n - lag)) / var
        if rho < inv_e:
            if lag > 1 and prev_rho > inv_e:
                return (lag - 1) + (prev_rho - inv_e) / (prev_rho - rho)
            return float(lag)
        prev_rho = rho
    return float(n // 2 - 1)


def independent_samples_per_second(t: Tau, seconds: float) -> float:
    """Independent samples per second: chains * n / (2 tau_int) / seconds."""
    return t.chains * t.n / (2.0 * t.tau) / seconds
