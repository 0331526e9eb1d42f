"""Effective sample size of a per-sweep observable series.

The reference writes only per-bin averages (equaltime_output); ESS needs the
per-sweep series, which the GPU driver reads with Dqmc.energy_all after each
sweep.  The integrated autocorrelation time uses the normalised
autocorrelation function (as auto_cor in lib/m_variance.f90:716-752) summed
with Sokal's self-consistent window (stop at the first lag M >= c * tau(M),
c = 5).  Independent chains share the same distribution, so the ACF is
averaged over chains before the window is applied; ESS of the whole batch is
(total samples) / (2 tau_int).
"""
from __future__ import annotations

import numpy as np


def acf(series: np.ndarray, max_lag: int | None = None) -> np.ndarray:
    """Normalised autocorrelation of x[chain, t], averaged over chains."""
    x = np.atleast_2d(np.asarray(series, float))
    n = x.shape[1]
    max_lag = n - 1 if max_lag is None else min(max_lag, n - 1)
    xc = x - x.mean(axis=1, keepdims=True)
    var = (xc * xc).mean()
    if var == 0.0:
        return np.ones(1)
    out = np.empty(max_lag + 1)
    for k in range(max_lag + 1):
        out[k] = (xc[:, : n - k] * xc[:, k:]).mean() / var
    return out


def tau_int(series: np.ndarray, c: float = 5.0) -> float:
    rho = acf(series)
    tau = 0.5
    for m in range(1, len(rho)):
        tau += rho[m]
        if m >= c * tau:
            break
    return max(tau, 0.5)


def ess(series: np.ndarray) -> tuple[float, float]:
    """(ESS, tau_int) of x[chain, t]."""
    x = np.atleast_2d(np.asarray(series, float))
    t = tau_int(x)
    return x.size / (2.0 * t), t


def double_occupancy(energy: np.ndarray, nsites: np.ndarray) -> np.ndarray:
    """D = Re(energy_bin(4) / energy_bin(1)) / N per chain (equaltime_measure zint_u)."""
    e = np.atleast_2d(energy)
    return (e[:, 3] / e[:, 0]).real / np.asarray(nsites, float)
