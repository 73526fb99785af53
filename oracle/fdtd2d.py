"""CPU oracle for the batched 2D TMz FDTD step — TEST INFRASTRUCTURE ONLY.

A vectorised NumPy restatement of ``BatchedFDTD2D`` in the reference
(``src/ceep/solvers/fdtd_2d_batched.py``), quirks included:

* interior H   (``:471-483``)   Hx on x in [n, nx-n), y in [n, ny-1);
                                Hy on x in [n, nx-1), y in [n, ny-n)
* H-CPML       (``:272-334``)   strips set  H = da*H +/- db*psi  on top of the
                                interior update (double update on the far side)
* interior E   (``:491-498``)   x in [n+1, nx-n), y in [n+1, ny-n)
* E-CPML       (``:336-406``)   strip cells get only  +/- dt/(eps_r eps0) * psi
* edge zeroing (``:503-507``), soft source (``:509-515``), probes (``:517-526``)

Where the reference loops over strip depth or columns in Python, this file
applies the same per-cell arithmetic as one array expression per strip; the
per-cell order of operations is the reference's, so the FP64 results agree to
rounding.

Keyword-only extensions (defaults reproduce the reference exactly):
``courant`` (c*dt/dx instead of the hard-coded 0.99/sqrt(2)), ``cpml_R0``,
``cpml_order``, ``waveform`` (an explicit per-step array) and ``dispersion``
(Debye / Lorentz ADE inside the interior-E region, composing
``src/ceep/materials/dispersive.py:240-426`` with ``src/ceep/solvers/fdtd_2d.py:163-178``).
"""
from __future__ import annotations

import math

import numpy as np

# src/ceep/core/constants.py:21-27
C_0 = 299_792_458.0
EPS_0 = 8.854187817e-12
MU_0 = 4.0 * math.pi * 1e-7
SOURCE_AMPLITUDE_SCALE = 1.049e10  # fdtd_2d_batched.py:177


def reference_dt_2d(dx: float) -> float:
    """``dt = dx / (C0 sqrt 2) * 0.99`` (fdtd_2d_batched.py:92)."""
    return dx / (C_0 * np.sqrt(2.0)) * 0.99


def gaussian_derivative_waveform(total_steps: int, dt: float, frequency: float,
                                 delay_factor: float = 5.0) -> np.ndarray:
    """Source waveform of fdtd_2d_batched.py:171-180 (FP64)."""
    tau = 1.0 / (2.0 * frequency)
    t0 = delay_factor * tau
    t_arr = np.arange(total_steps) * dt
    w = -(t_arr - t0) / tau * np.exp(-((t_arr - t0) / tau) ** 2)
    return w * SOURCE_AMPLITUDE_SCALE


def cpml_profile(n: int, dx: float, dt: float, R: float = 1e-8, m: int = 3):
    """Graded CPML ``b``/``c`` of fdtd_2d_batched.py:195-238 (FP64)."""
    eta_0 = np.sqrt(MU_0 / EPS_0)
    d_pml = n * dx
    sigma_max = -(m + 1) * np.log(R) / (2.0 * eta_0 * d_pml)
    d = np.arange(n, dtype=np.float64)
    sigma = sigma_max * ((n - 1 - d) / (n - 1)) ** m
    b = np.exp(-sigma * dt / EPS_0)
    return b, b - 1.0


def ade_coefficients(dt, debye=(), lorentz=(), shape=None):
    """Per-cell ADE coefficients, dispersive.py:240-339.

    ``debye``  : sequence of (delta_eps, tau) maps
    ``lorentz``: sequence of (delta_eps, omega_0, delta) maps
    Returns (eps_eff_add, [(k1, k2, gamma)] for Debye, [(k1, k2, k3)] for Lorentz).
    """
    eps_add = np.zeros(shape)
    deb = []
    for de, tau in debye:
        de = np.broadcast_to(np.asarray(de, np.float64), shape)
        tau = np.broadcast_to(np.asarray(tau, np.float64), shape)
        k1 = np.zeros(shape); k2 = np.zeros(shape); g = np.zeros(shape)
        valid = tau > 0
        denom = 2.0 * tau[valid] + dt
        k1[valid] = (2.0 * tau[valid] - dt) / denom
        k2[valid] = (2.0 * EPS_0 * de[valid] * dt) / denom
        g[valid] = (1.0 + k1[valid]) / 2.0
        eps_add[valid] += k2[valid] / 2.0
        deb.append((k1, k2, g))
    lor = []
    for de, w0, dl in lorentz:
        de = np.broadcast_to(np.asarray(de, np.float64), shape)
        w0 = np.broadcast_to(np.asarray(w0, np.float64), shape)
        dl = np.broadcast_to(np.asarray(dl, np.float64), shape)
        k1 = np.zeros(shape); k2 = np.zeros(shape); k3 = np.zeros(shape)
        valid = w0 > 0
        d = dl[valid]
        w02 = w0[valid] ** 2
        dt2 = dt * dt
        denom = 4.0 + 2.0 * d * dt + w02 * dt2
        k1[valid] = (8.0 - 2.0 * w02 * dt2) / denom
        k3[valid] = -(4.0 - 2.0 * d * dt + w02 * dt2) / denom
        k2[valid] = 2.0 * EPS_0 * de[valid] * w02 * dt2 / denom
        eps_add[valid] += k2[valid] / 2.0
        lor.append((k1, k2, k3))
    return eps_add, deb, lor


class Fdtd2DOracle:
    """Batched 2D TMz oracle.  State arrays use the reference layout (B, nx, ny)."""

    def __init__(self, nx, ny, dx, total_steps, cpml_thickness, source_positions,
                 probe_positions, frequency, delay_factor=5.0, *, eps_r=None,
                 sigma_e=None, dtype=np.float64, courant=None, cpml_R0=1e-8,
                 cpml_order=3, waveform=None, dispersion=None):
        self.nx, self.ny, self.dx = int(nx), int(ny), float(dx)
        self.total_steps = int(total_steps)
        self.n = int(cpml_thickness)
        self.src = [tuple(int(v) for v in p) for p in source_positions]
        self.prb = [tuple(int(v) for v in p) for p in probe_positions]
        self.frequency = float(frequency)
        self.B = len(self.src)
        self.dtype = np.dtype(dtype)
        if courant is None:
            self.dt = reference_dt_2d(dx)
        else:
            self.dt = float(courant) * dx / C_0
        self.eps_r = np.ones((nx, ny)) if eps_r is None else np.array(eps_r, np.float64)
        self.sigma_e = np.zeros((nx, ny)) if sigma_e is None else np.array(sigma_e, np.float64)
        if waveform is None:
            waveform = gaussian_derivative_waveform(self.total_steps, self.dt,
                                                    self.frequency, delay_factor)
        self.waveform = np.asarray(waveform, np.float64)
        self.R0, self.order = cpml_R0, cpml_order
        self.dispersion = dispersion or {}
        self._build()

    # -- coefficients (fdtd_2d_batched.py:151-167, :195-238) -----------------
    def _build(self):
        nx, ny, dt, B, n = self.nx, self.ny, self.dt, self.B, self.n
        dtp = self.dtype
        shape = (nx, ny)
        eps_add, self.deb, self.lor = ade_coefficients(
            dt, self.dispersion.get("debye", ()), self.dispersion.get("lorentz", ()), shape)
        eps = self.eps_r * EPS_0 + eps_add
        s = self.sigma_e * dt / (2.0 * eps)
        self.ca = ((1.0 - s) / (1.0 + s)).astype(dtp)
        self.cb = ((dt / eps) / (1.0 + s)).astype(dtp)
        self.db = dtp.type(dt / MU_0)
        # E-CPML uses eps_r only, no sigma and no ADE (fdtd_2d_batched.py:348)
        self.dt_eps = (dt / (self.eps_r * EPS_0)).astype(dtp)
        if n > 0:
            b, c = cpml_profile(n, self.dx, dt, self.R0, self.order)
        else:
            b = c = np.zeros(0)
        self.b, self.c = b.astype(dtp), c.astype(dtp)
        z = lambda *s_: np.zeros(s_, dtp)
        self.ez, self.hx, self.hy = z(B, nx, ny), z(B, nx, ny), z(B, nx, ny)
        self.psi_hxy_lo, self.psi_hxy_hi = z(B, n, ny), z(B, n, ny)
        self.psi_ezx_lo, self.psi_ezx_hi = z(B, n, ny), z(B, n, ny)
        self.psi_hyx_lo, self.psi_hyx_hi = z(B, nx, n), z(B, nx, n)
        self.psi_ezy_lo, self.psi_ezy_hi = z(B, nx, n), z(B, nx, n)
        self.j_deb = [z(B, nx, ny) for _ in self.deb]
        self.j_lor = [z(B, nx, ny) for _ in self.lor]
        self.j_lor_prev = [z(B, nx, ny) for _ in self.lor]
        self.deb = [tuple(a.astype(dtp) for a in t) for t in self.deb]
        self.lor = [tuple(a.astype(dtp) for a in t) for t in self.lor]
        self.probe_data = np.zeros((B, len(self.prb), self.total_steps), dtp)
        self.step_index = 0

    # -- one time step -------------------------------------------------------
    def step(self):
        nx, ny, n = self.nx, self.ny, self.n
        inv_dx = 1.0 / self.dx
        inv_dy = inv_dx
        ez, hx, hy = self.ez, self.hx, self.hy
        db, b, c = self.db, self.b, self.c
        t = self.dtype.type

        # interior H, fdtd_2d_batched.py:471-483 (da == 1 exactly in 2D)
        hx[:, n:nx - n, n:ny - 1] = hx[:, n:nx - n, n:ny - 1] - db * t(inv_dy) * (
            ez[:, n:nx - n, n + 1:ny] - ez[:, n:nx - n, n:ny - 1])
        hy[:, n:nx - 1, n:ny - n] = hy[:, n:nx - 1, n:ny - n] + db * t(inv_dx) * (
            ez[:, n + 1:nx, n:ny - n] - ez[:, n:nx - 1, n:ny - n])

        if n > 0:
            # H-CPML x strips on Hy, fdtd_2d_batched.py:282-311
            d = (ez[:, 1:n + 1, :] - ez[:, 0:n, :]) * t(inv_dx)
            self.psi_hxy_lo[:] = b[None, :, None] * self.psi_hxy_lo + c[None, :, None] * d
            hy[:, 0:n, :] = hy[:, 0:n, :] + db * self.psi_hxy_lo
            x0 = nx - n
            d = (ez[:, x0 + 1:nx, :] - ez[:, x0:nx - 1, :]) * t(inv_dx)
            br, cr = b[::-1][:n - 1], c[::-1][:n - 1]
            self.psi_hxy_hi[:, :n - 1] = br[None, :, None] * self.psi_hxy_hi[:, :n - 1] + cr[None, :, None] * d
            hy[:, x0:nx - 1, :] = hy[:, x0:nx - 1, :] + db * self.psi_hxy_hi[:, :n - 1]
            # H-CPML y strips on Hx, fdtd_2d_batched.py:313-334
            d = (ez[:, :, 1:n + 1] - ez[:, :, 0:n]) * t(inv_dy)
            self.psi_hyx_lo[:] = b[None, None, :] * self.psi_hyx_lo + c[None, None, :] * d
            hx[:, :, 0:n] = hx[:, :, 0:n] - db * self.psi_hyx_lo
            y0 = ny - n
            d = (ez[:, :, y0 + 1:ny] - ez[:, :, y0:ny - 1]) * t(inv_dy)
            self.psi_hyx_hi[:, :, :n - 1] = br[None, None, :] * self.psi_hyx_hi[:, :, :n - 1] + cr[None, None, :] * d
            hx[:, :, y0:ny - 1] = hx[:, :, y0:ny - 1] - db * self.psi_hyx_hi[:, :, :n - 1]

        # interior E, fdtd_2d_batched.py:491-498
        I = (slice(None), slice(n + 1, nx - n), slice(n + 1, ny - n))
        Im = (slice(None), slice(n, nx - n - 1), slice(n + 1, ny - n))
        Jm = (slice(None), slice(n + 1, nx - n), slice(n, ny - n - 1))
        ez_old = ez[I].copy()
        ez[I] = self.ca[None, n + 1:nx - n, n + 1:ny - n] * ez[I] + self.cb[None, n + 1:nx - n, n + 1:ny - n] * (
            (hy[I] - hy[Im]) * t(inv_dx) - (hx[I] - hx[Jm]) * t(inv_dy))
        if self.deb or self.lor:
            self._ade(I, ez_old)

        if n > 0:
            de = self.dt_eps
            # E-CPML x strips, fdtd_2d_batched.py:355-378 (columns 1..n and nx-n..nx-1, rows >= 1)
            d = (hy[:, 1:n + 1, 1:] - hy[:, 0:n, 1:]) * t(inv_dx)
            self.psi_ezx_lo[:, :, 1:] = b[None, :, None] * self.psi_ezx_lo[:, :, 1:] + c[None, :, None] * d
            ez[:, 1:n + 1, 1:] = ez[:, 1:n + 1, 1:] + de[None, 1:n + 1, 1:] * self.psi_ezx_lo[:, :, 1:]
            x0 = nx - n
            d = (hy[:, x0:nx, 1:] - hy[:, x0 - 1:nx - 1, 1:]) * t(inv_dx)
            self.psi_ezx_hi[:, :, 1:] = b[::-1][None, :, None] * self.psi_ezx_hi[:, :, 1:] + c[::-1][None, :, None] * d
            ez[:, x0:nx, 1:] = ez[:, x0:nx, 1:] + de[None, x0:nx, 1:] * self.psi_ezx_hi[:, :, 1:]
            # E-CPML y strips, fdtd_2d_batched.py:380-406 (rows 1..n and ny-n..ny-1, columns >= 1)
            d = (hx[:, 1:, 1:n + 1] - hx[:, 1:, 0:n]) * t(inv_dy)
            self.psi_ezy_lo[:, 1:, :] = b[None, None, :] * self.psi_ezy_lo[:, 1:, :] + c[None, None, :] * d
            ez[:, 1:, 1:n + 1] = ez[:, 1:, 1:n + 1] - de[None, 1:, 1:n + 1] * self.psi_ezy_lo[:, 1:, :]
            y0 = ny - n
            d = (hx[:, 1:, y0:ny] - hx[:, 1:, y0 - 1:ny - 1]) * t(inv_dy)
            self.psi_ezy_hi[:, 1:, :] = b[::-1][None, None, :] * self.psi_ezy_hi[:, 1:, :] + c[::-1][None, None, :] * d
            ez[:, 1:, y0:ny] = ez[:, 1:, y0:ny] - de[None, 1:, y0:ny] * self.psi_ezy_hi[:, 1:, :]

        # edges, source, probes: fdtd_2d_batched.py:503-526
        ez[:, 0, :] = 0
        ez[:, -1, :] = 0
        ez[:, :, 0] = 0
        ez[:, :, -1] = 0
        s = self.step_index
        w = self.dtype.type(self.waveform[s])
        for bb, (sx, sy) in enumerate(self.src):
            ez[bb, sx, sy] += w
        for p, (px, py) in enumerate(self.prb):
            self.probe_data[:, p, s] = ez[:, px, py]
        self.step_index += 1

    def _ade(self, I, ez_old):
        """ADE inside the interior-E region (dispersive.py:341-404, fdtd_2d.py:163-178)."""
        ez = self.ez
        sl = I[1:]
        cb = self.cb[None][(slice(None),) + sl]
        sum_gj = 0.0
        for (k1, k2, g), J in zip(self.deb, self.j_deb):
            sum_gj = sum_gj + g[None][(slice(None),) + sl] * J[I]
        for (k1, k2, k3), J in zip(self.lor, self.j_lor):
            sum_gj = sum_gj + J[I]  # gamma == 1 for Lorentz (dispersive.py:297)
        ez[I] = ez[I] - cb * sum_gj
        de_dt = (ez[I] - ez_old) / self.dtype.type(self.dt)
        for (k1, k2, g), J in zip(self.deb, self.j_deb):
            J[I] = k1[None][(slice(None),) + sl] * J[I] + k2[None][(slice(None),) + sl] * de_dt
        for (k1, k2, k3), J, Jp in zip(self.lor, self.j_lor, self.j_lor_prev):
            j_new = (k1[None][(slice(None),) + sl] * J[I] + k3[None][(slice(None),) + sl] * Jp[I]
                     + k2[None][(slice(None),) + sl] * de_dt)
            Jp[I] = J[I]
            J[I] = j_new

    def run(self, steps=None):
        steps = self.total_steps - self.step_index if steps is None else steps
        for _ in range(steps):
            self.step()
        return self.probe_data


def run_cpu_oracle(nx, ny, dx, total_steps, source_positions, probe_positions,
                   frequency, delay_factor=5.0, eps_r=None, sigma_e=None):
    """Restates ``BatchedFDTD2D.run_cpu`` (fdtd_2d_batched.py:540-611): no CPML,
    full-domain update, H zeroed on the far edge, E zeroed on all edges."""
    B = len(source_positions)
    dt = reference_dt_2d(dx)
    eps_r = np.ones((nx, ny)) if eps_r is None else np.asarray(eps_r, np.float64)
    sigma_e = np.zeros((nx, ny)) if sigma_e is None else np.asarray(sigma_e, np.float64)
    eps = eps_r * EPS_0
    s = sigma_e * dt / (2.0 * eps)
    ca = ((1.0 - s) / (1.0 + s))[None]
    cb = ((dt / eps) / (1.0 + s))[None]
    db = dt / MU_0
    inv = 1.0 / dx
    w = gaussian_derivative_waveform(total_steps, dt, frequency, delay_factor)
    ez = np.zeros((B, nx, ny)); hx = np.zeros_like(ez); hy = np.zeros_like(ez)
    out = np.zeros((B, len(probe_positions), total_steps))
    for st in range(total_steps):
        hx[:, :, :-1] = hx[:, :, :-1] - db * inv * (ez[:, :, 1:] - ez[:, :, :-1])
        hy[:, :-1, :] = hy[:, :-1, :] + db * inv * (ez[:, 1:, :] - ez[:, :-1, :])
        hx[:, :, -1] = 0
        hy[:, -1, :] = 0
        ez[:, 1:, 1:] = ca[:, 1:, 1:] * ez[:, 1:, 1:] + cb[:, 1:, 1:] * (
            (hy[:, 1:, 1:] - hy[:, :-1, 1:]) * inv - (hx[:, 1:, 1:] - hx[:, 1:, :-1]) * inv)
        ez[:, 0, :] = 0; ez[:, -1, :] = 0; ez[:, :, 0] = 0; ez[:, :, -1] = 0
        for bb, (sx, sy) in enumerate(source_positions):
            ez[bb, sx, sy] += w[st]
        for p, (px, py) in enumerate(probe_positions):
            out[:, p, st] = ez[:, px, py]
    return out
