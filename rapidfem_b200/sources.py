"""Waveforms of driven runs and their discretisations on the device paths.

* `gaussian_pulse` is the reference's GaussianPulse (session.rs:242-261):
  g(t) = exp(-((t - t0)/tau)^2) cos(2 pi f0 (t - t0)).
* `gaussian_sine` is the Gaussian-modulated sine of the stiff driven
  configuration: g(t) = exp(-(t - t0)^2 / (2 sigma^2)) sin(2 pi f0 (t - t0)).
* `lserk_stage_times` gives the stage abscissae c_s of the LSERK4 scheme
  (explicit.rs:100-135 with the Carpenter-Kennedy coefficients of
  constants.rs:106-122), for sampling a waveform at the stage times
  (dgtd_run_lserk_stages / dgtd_transient_f64_stages).
* `step_polynomial` fits a waveform over one exponential step with a
  polynomial (Chebyshev interpolation) and returns its monomial coefficients
  about the step start, the source of dgtd_etd_step_poly / dgtd_etd_try.
"""
from __future__ import annotations

import numpy as np

LSERK_A = (0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
           -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0)
LSERK_B = (1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
           1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
           2277821191437.0 / 14882151754819.0)


def lserk_stage_times() -> np.ndarray:
    """c[5]: stage s of a step from t evaluates the RHS at t + c[s] h
    (c_0 = 0, w_0 = 1, c_{s+1} = c_s + b_s w_s, w_{s+1} = a_{s+1} w_s + 1)."""
    c = np.zeros(5)
    w = 1.0
    for s in range(4):
        c[s + 1] = c[s] + LSERK_B[s] * w
        w = LSERK_A[s + 1] * w + 1.0
    return c


def gaussian_pulse(t, t0, tau, f0=0.0):
    t = np.asarray(t, dtype=np.float64)
    env = np.exp(-((t - t0) / tau) ** 2)
    return env * np.cos(2 * np.pi * f0 * (t - t0)) if f0 else env


def gaussian_sine(t, t0, sigma_t, f0):
    t = np.asarray(t, dtype=np.float64)
    return np.exp(-((t - t0) ** 2) / (2 * sigma_t ** 2)) * np.sin(2 * np.pi * f0 * (t - t0))


def stage_samples(g, t0: float, h: float, steps: int) -> np.ndarray:
    """g at the stage times of `steps` LSERK4 steps of h from t0: [5*steps]."""
    c = lserk_stage_times()
    t = t0 + h * (np.arange(steps)[:, None] + c[None, :])
    return np.asarray(g(t.ravel()), dtype=np.float64)


def step_polynomial(g, t: float, h: float, n_coef: int = 8):
    """(coef, err): monomial coefficients of the degree n_coef-1 interpolant of g
    at the Chebyshev points of [t, t+h], about t (g(t+tau) ~ sum coef[k] tau^k),
    and the largest deviation from g at the midpoints between those points."""
    k = np.arange(n_coef)
    x = np.cos((2 * k + 1) * np.pi / (2 * n_coef))          # Chebyshev points on [-1, 1]
    tau = 0.5 * h * (x + 1.0)
    vals = np.asarray(g(t + tau), dtype=np.float64)
    # interpolant in the scaled variable s = tau / h, then back to tau
    s = tau / h
    vander = np.vander(s, n_coef, increasing=True)
    cs = np.linalg.solve(vander, vals)
    coef = cs / h ** k
    xm = np.cos(np.arange(n_coef + 1) * np.pi / n_coef)
    sm = 0.5 * (xm + 1.0)
    err = float(np.max(np.abs(np.polyval(cs[::-1], sm) - g(t + h * sm))))
    return coef, err

