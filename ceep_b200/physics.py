"""Host-side FP64 precompute of every coefficient the kernels consume.

All transcendental work (exp, log, sin, cos) happens here in NumPy FP64 and is
rounded to FP32 once, so the device code is pure FMA arithmetic.
"""
from __future__ import annotations

import numpy as np

from .constants import C_0, EPS_0, MU_0, ETA_0, SOURCE_AMPLITUDE_SCALE


def gaussian_derivative(total_steps: int, dt: float, frequency: float, delay_factor: float = 5.0) -> np.ndarray:
    """Reference source waveform: fdtd_2d_batched.py:171-180 / fdtd_3d_batched.py:305-313."""
    tau = 1.0 / (2.0 * frequency)
    t0 = delay_factor * tau
    t = np.arange(total_steps) * dt
    return -(t - t0) / tau * np.exp(-((t - t0) / tau) ** 2) * SOURCE_AMPLITUDE_SCALE


def modulated_gaussian(total_steps: int, dt: float, frequency: float, tau: float = 0.3e-9,
                       t0: float | None = None, amplitude: float = 1.0) -> np.ndarray:
    """Gaussian-modulated sinusoid exp(-((t-t0)/tau)^2) sin(2 pi f (t-t0)), t0 = 4 tau by default."""
    t0 = 4.0 * tau if t0 is None else t0
    t = np.arange(total_steps) * dt
    return amplitude * np.exp(-((t - t0) / tau) ** 2) * np.sin(2.0 * np.pi * frequency * (t - t0))


def cpml_profile(n: int, dx: float, dt: float, R0: float = 1e-8, order: int = 3):
    """Polynomially graded CPML b = exp(-sigma dt / eps0), c = b - 1
    (fdtd_2d_batched.py:195-238; index 0 is the outermost cell)."""
    if n == 0:
        return np.zeros(0), np.zeros(0)
    sigma_max = -(order + 1) * np.log(R0) / (2.0 * ETA_0 * n * dx)
    d = np.arange(n, dtype=np.float64)
    sigma = sigma_max * ((n - 1 - d) / (n - 1)) ** order
    b = np.exp(-sigma * dt / EPS_0)
    return b, b - 1.0


def ade_coefficients(dt: float, debye=(), lorentz=(), shape=None):
    """Per-cell ADE coefficients (dispersive.py:240-339).

    debye   : sequence of (delta_eps, tau) maps (scalars broadcast)
    lorentz : sequence of (delta_eps, omega_0, delta) maps
    Returns eps_add (F/m, added to eps_inf*eps0) and a (poles, *shape, 4) array
    holding Debye (k1, k2, gamma, 0) then Lorentz (k1, k2, k3, 0).
    """
    poles = len(debye) + len(lorentz)
    eps_add = np.zeros(shape)
    out = np.zeros((poles,) + tuple(shape) + (4,))
    q = 0
    for de, tau in debye:
        de = np.broadcast_to(np.asarray(de, np.float64), shape)
        tau = np.broadcast_to(np.asarray(tau, np.float64), shape)
        v = tau > 0
        den = 2.0 * tau[v] + dt
        k1 = (2.0 * tau[v] - dt) / den
        k2 = (2.0 * EPS_0 * de[v] * dt) / den
        out[q][v, 0] = k1
        out[q][v, 1] = k2
        out[q][v, 2] = (1.0 + k1) / 2.0
        eps_add[v] += k2 / 2.0
        q += 1
    for de, w0, dl in lorentz:
        de = np.broadcast_to(np.asarray(de, np.float64), shape)
        w0 = np.broadcast_to(np.asarray(w0, np.float64), shape)
        dl = np.broadcast_to(np.asarray(dl, np.float64), shape)
        v = w0 > 0
        d, w02, dt2 = dl[v], w0[v] ** 2, dt * dt
        den = 4.0 + 2.0 * d * dt + w02 * dt2
        k2 = 2.0 * EPS_0 * de[v] * w02 * dt2 / den
        out[q][v, 0] = (8.0 - 2.0 * w02 * dt2) / den
        out[q][v, 1] = k2
        out[q][v, 2] = -(4.0 - 2.0 * d * dt + w02 * dt2) / den
        eps_add[v] += k2 / 2.0
        q += 1
    return eps_add, out


def update_coefficients(eps_r, sigma_e, dt, eps_add=None):
    """ca, cb of fdtd_2d_batched.py:151-167 (grid.py:174-189 when eps_add is given)."""
    eps = np.asarray(eps_r, np.float64) * EPS_0
    if eps_add is not None:
        eps = eps + eps_add
    s = np.asarray(sigma_e, np.float64) * dt / (2.0 * eps)
    return (1.0 - s) / (1.0 + s), (dt / eps) / (1.0 + s)


def dft_twiddles(frequencies, nsteps: int, dt: float) -> np.ndarray:
    """(F, T, 2) float32: (cos(w n dt) dt, -sin(w n dt) dt), the running-DFT
    weights of dft.py:75-90, evaluated in FP64 (no FP32 phase accumulation)."""
    w = 2.0 * np.pi * np.asarray(frequencies, np.float64)
    ph = np.outer(w, np.arange(nsteps) * dt)
    return np.stack([np.cos(ph) * dt, -np.sin(ph) * dt], axis=-1).astype(np.float32)


__all__ = ["gaussian_derivative", "modulated_gaussian", "cpml_profile", "ade_coefficients",
           "update_coefficients", "dft_twiddles", "C_0", "EPS_0", "MU_0"]
