"""Integrated autocorrelation time and effective sample size of chain series.

The reference reports only a 10-block standard error
(src/number_conserving/benchmarks/compare.py:86-124); the effective sample
size needs tau_int, estimated here two ways on [chains, samples] arrays:

* windowed autocorrelation, averaged over independent chains, with Sokal's
  self-consistent window (smallest W with W >= c * tau_int(W), c = 5);
* blocking: the variance of block means grows as 2 tau_int / block length.
"""
from __future__ import annotations

import numpy as np


def autocorr(series: np.ndarray, max_lag: int) -> np.ndarray:
    """Normalised autocorrelation rho(t), t = 0..max_lag, pooled over chains.

    series: [chains, samples]; each chain is centred on the ensemble mean of
    its time index-independent average (chains are independent and share a
    stationary distribution)."""
    x = np.asarray(series, dtype=np.float64)
    if x.ndim == 1:
        x = x[None, :]
    x = x - x.mean()
    s = x.shape[1]
    max_lag = min(max_lag, s - 1)
    c0 = np.mean(x * x)
    if c0 == 0.0:
        return np.concatenate([[1.0], np.zeros(max_lag)])
    rho = np.empty(max_lag + 1)
    for t in range(max_lag + 1):
        rho[t] = np.mean(x[:, : s - t] * x[:, t:]) / c0
    return rho


def tau_int(series: np.ndarray, c: float = 5.0) -> tuple[float, int]:
    """(tau_int, window) with tau_int = 1/2 + sum_{t=1}^{W} rho(t)."""
    x = np.asarray(series, dtype=np.float64)
    s = x.shape[-1]
    rho = autocorr(x, s // 2)
    tau = 0.5
    for w in range(1, len(rho)):
        tau += rho[w]
        if w >= c * tau:
            return float(tau), w
    return float(tau), len(rho) - 1


def tau_blocking(series: np.ndarray, block: int) -> float:
    """tau_int from the variance of block means of length `block`."""
    x = np.asarray(series, dtype=np.float64)
    if x.ndim == 1:
        x = x[None, :]
    nb = x.shape[1] // block
    if nb < 2:
        raise ValueError("need at least two blocks")
    means = x[:, : nb * block].reshape(x.shape[0], nb, block).mean(axis=2)
    var = np.var(x - x.mean(axis=1, keepdims=True))
    if var == 0.0:
        return 0.5
    return float(0.5 * block * np.var(means - means.mean(axis=1, keepdims=True), ddof=0) / var * nb / (nb - 1))


def ess_per_second(samples_per_second: float, taus: dict) -> tuple[float, str]:
    """ESS/s = samples/s / (2 max tau): the minimum over the observables."""
    name = max(taus, key=lambda k: taus[k])
    return samples_per_second / (2.0 * taus[name]), name
