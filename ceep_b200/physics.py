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


def _f64(a, device):
    import torch
    if isinstance(a, torch.Tensor):
        return a.to(device=device if device is not None else a.device, dtype=torch.float64)
    return torch.as_tensor(np.asarray(a, np.float64)).to(device)


def ade_tensors(dt: float, debye=(), lorentz=(), shape=None, device=None):
    """ade_coefficients evaluated with torch in FP64 on `device`: every
    expression is the NumPy one above with the same operation order (one
    IEEE-rounded op per torch call, no fusion), so the maps are bit-identical.
    Returns eps_add and a (poles, *shape, 4) FP64 tensor."""
    import torch
    bc = lambda a: torch.broadcast_to(_f64(a, device), shape)
    eps_add = torch.zeros(shape, dtype=torch.float64, device=device)
    zero = torch.zeros((), dtype=torch.float64, device=device)
    poles = []
    for de, tau in debye:
        de, tau = bc(de), bc(tau)
        v = tau > 0
        den = 2.0 * tau + dt
        k1 = (2.0 * tau - dt) / den
        k2 = (2.0 * EPS_0 * de * dt) / den
        poles.append(torch.stack([torch.where(v, k1, zero), torch.where(v, k2, zero),
                                  torch.where(v, (1.0 + k1) / 2.0, zero), torch.zeros_like(k1)], -1))
        eps_add = torch.where(v, eps_add + k2 / 2.0, eps_add)
    for de, w0, dl in lorentz:
        de, w0, d = bc(de), bc(w0), bc(dl)
        v = w0 > 0
        w02, dt2 = w0 * w0, dt * dt
        den = 4.0 + 2.0 * d * dt + w02 * dt2
        k2 = 2.0 * EPS_0 * de * w02 * dt2 / den
        k1 = (8.0 - 2.0 * w02 * dt2) / den
        k3 = -(4.0 - 2.0 * d * dt + w02 * dt2) / den
        poles.append(torch.stack([torch.where(v, k1, zero), torch.where(v, k2, zero),
                                  torch.where(v, k3, zero), torch.zeros_like(k1)], -1))
        eps_add = torch.where(v, eps_add + k2 / 2.0, eps_add)
    ade = torch.stack(poles) if poles else torch.zeros((0,) + tuple(shape) + (4,), dtype=torch.float64,
                                                       device=device)
    return eps_add, ade


def rdiv(num: float, t):
    """num / t elementwise with one correctly rounded division, as NumPy's
    scalar / array.  torch evaluates float / Tensor as reciprocal(t) * num,
    two roundings that differ from the quotient by an ulp in about a quarter
    of FP64 elements.  The numerator is a 0-d tensor filled on t's device (no
    host-to-device copy, so no wait for the stream)."""
    import torch
    return torch.div(t.new_full((), num), t)


def coefficient_tensors(eps_r, sigma_e, dt: float, debye=(), lorentz=(), device=None):
    """2D: ade_coefficients + update_coefficients on the device (see
    ade_tensors), in the kernel layout: coef (ny, nx, 4) float32 = (ca, cb,
    dt/(eps_r eps0), 0) and ade (poles, ny, nx, 4) float32.  Only the (nx, ny)
    FP64 maps cross the host link."""
    import torch
    eps_r = _f64(eps_r, device)
    eps_add, ade = ade_tensors(dt, debye, lorentz, eps_r.shape, eps_r.device)
    eps = eps_r * EPS_0
    if ade.shape[0]:
        eps = eps + eps_add
    s = torch.broadcast_to(_f64(sigma_e, eps_r.device), eps_r.shape) * dt / (2.0 * eps)
    ca, cb = (1.0 - s) / (1.0 + s), rdiv(dt, eps) / (1.0 + s)
    dteps = rdiv(dt, eps_r * EPS_0)
    coef = torch.stack([ca.t(), cb.t(), dteps.t(), torch.zeros_like(ca).t()], -1).float().contiguous()
    return coef, ade.transpose(1, 2).float().contiguous()


def coefficient_tensors_kernel(eps_r, sigma_e, dt: float, debye=(), lorentz=(), device=None):
    """The maps of coefficient_tensors from one library kernel
    (``ceep2d_material_coefficients``: the same FP64 operations in the same
    order, no contraction, so the same bits) instead of a chain of torch
    element-wise launches; the solver's material update uses this one."""
    import ctypes as C
    import torch
    from ._lib import check, lib
    eps = _f64(eps_r, device)
    dev, shape = eps.device, tuple(eps.shape)
    full = lambda a: torch.broadcast_to(_f64(a, dev), shape).contiguous()
    sig = full(sigma_e)
    maps = [full(a) for p in debye for a in p] + [full(a) for p in lorentz for a in p]
    nx, ny = shape
    npoles = len(debye) + len(lorentz)
    coef = torch.empty((ny, nx, 4), dtype=torch.float32, device=dev)
    ade = torch.empty((npoles, ny, nx, 4), dtype=torch.float32, device=dev)
    ptrs = (C.c_void_p * max(1, len(maps)))(*[m.data_ptr() for m in maps])
    check(lib().ceep2d_material_coefficients(eps.contiguous().data_ptr(), sig.data_ptr(), ptrs, len(debye),
                                             len(lorentz), nx, ny, float(dt), EPS_0, coef.data_ptr(),
                                             ade.data_ptr() if npoles else None,
                                             torch.cuda.current_stream(dev).cuda_stream),
          "ceep2d_material_coefficients")
    return coef, ade


def coefficient_tensors_3d(eps_r, sigma_e, mu_r, sigma_m, dt: float, debye=(), lorentz=(), device=None):
    """3D (fdtd_3d_batched.py:281-296 with the ADE eps): coef (nz, ny, nx, 4)
    float32 = (da, db, ca, cb) and ade (poles, nz, ny, nx, 4) float32 from
    (nx, ny, nz) FP64 maps, on the device with the host formulas' operation order."""
    import torch
    eps_r = _f64(eps_r, device)
    dev, shp = eps_r.device, eps_r.shape
    bc = lambda a: torch.broadcast_to(_f64(a, dev), shp)
    eps_add, ade = ade_tensors(dt, debye, lorentz, shp, dev)
    eps = eps_r * EPS_0 + eps_add
    mu = bc(mu_r) * MU_0
    se = bc(sigma_e) * dt / (2.0 * eps)
    sm = bc(sigma_m) * dt / (2.0 * mu)
    ca, cb = (1.0 - se) / (1.0 + se), rdiv(dt, eps) / (1.0 + se)
    da, db = (1.0 - sm) / (1.0 + sm), rdiv(dt, mu) / (1.0 + sm)
    coef = torch.stack([da, db, ca, cb], -1).permute(2, 1, 0, 3).float().contiguous()
    return coef, ade.permute(0, 3, 2, 1, 4).float().contiguous()


def dft_twiddles(frequencies, nsteps: int, dt: float) -> np.ndarray:
    """(F, T, 2) float32: (cos(w n dt) dt, -sin(w n dt) dt), the running-DFT
    weights of dft.py:75-90, evaluated in FP64 (no FP32 phase accumulation)."""
    w = 2.0 * np.pi * np.asarray(frequencies, np.float64)
    ph = np.outer(w, np.arange(nsteps) * dt)
    return np.stack([np.cos(ph) * dt, -np.sin(ph) * dt], axis=-1).astype(np.float32)


__all__ = ["gaussian_derivative", "modulated_gaussian", "cpml_profile", "ade_coefficients",
           "update_coefficients", "ade_tensors", "coefficient_tensors", "coefficient_tensors_kernel",
           "coefficient_tensors_3d", "dft_twiddles",
           "C_0", "EPS_0", "MU_0"]
