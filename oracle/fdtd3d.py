"""CPU oracle for the batched 3D Yee FDTD step — TEST INFRASTRUCTURE ONLY.

Vectorised NumPy restatement of ``BatchedFDTD3D`` in the reference
(``src/ceep/solvers/fdtd_3d_batched.py``):

* dt = cfl_timestep_3d(dx, dx, dx, 0.5) * 0.99           (:133, constants.py:143-175)
* ca, cb, da, db including sigma_m                        (:281-296)
* interior H boxes                                        (:753-818)
* H-CPML on x, then y, then z faces; the far faces use backward differences
  and every face recurrence runs over the whole slab      (:398-586)
* interior E only on [n+1, N-n)^3                         (:820-884)
* E zeroed on the three LOW faces only                    (:936-944)
* soft Ez source, Ez probes                               (:949-958)
* compute_energy                                          (:987-1011)

The never-called ``*_deprecated`` E-CPML functions (:588-751) are not part of
the path and are not restated.  State arrays use the reference layout
(B, nx, ny, nz).
"""
from __future__ import annotations

import math

import numpy as np

from .fdtd2d import C_0, EPS_0, MU_0, cpml_profile, gaussian_derivative_waveform, ade_coefficients


def reference_dt_3d(dx: float) -> float:
    dt_max = 1.0 / (C_0 * math.sqrt(1.0 / (dx * dx) + 1.0 / (dx * dx) + 1.0 / (dx * dx)))
    return 0.5 * dt_max * 0.99


class Fdtd3DOracle:
    def __init__(self, nx, ny, nz, dx, total_steps, cpml_thickness, source_positions,
                 probe_positions, frequency, delay_factor=5.0, *, eps_r=None, sigma_e=None,
                 mu_r=None, sigma_m=None, dtype=np.float64, waveform=None, dispersion=None,
                 cpml_R0=1e-8, cpml_order=3):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dx = float(dx)
        self.total_steps = int(total_steps)
        self.n = int(cpml_thickness)
        self.src = [tuple(int(v) for v in p) for p in source_positions]
        self.prb = [tuple(int(v) for v in p) for p in probe_positions]
        self.B = len(self.src)
        self.dtype = np.dtype(dtype)
        self.dt = reference_dt_3d(dx)
        shp = (nx, ny, nz)
        self.eps_r = np.ones(shp) if eps_r is None else np.array(eps_r, np.float64)
        self.sigma_e = np.zeros(shp) if sigma_e is None else np.array(sigma_e, np.float64)
        self.mu_r = np.ones(shp) if mu_r is None else np.array(mu_r, np.float64)
        self.sigma_m = np.zeros(shp) if sigma_m is None else np.array(sigma_m, np.float64)
        if waveform is None:
            waveform = gaussian_derivative_waveform(self.total_steps, self.dt, frequency, delay_factor)
        self.waveform = np.asarray(waveform, np.float64)
        self.dispersion = dispersion or {}
        self.R0, self.order = cpml_R0, cpml_order
        self._build()

    def _build(self):
        B, nx, ny, nz, n, dt = self.B, self.nx, self.ny, self.nz, self.n, self.dt
        dtp = self.dtype
        shp = (nx, ny, nz)
        eps_add, deb, lor = ade_coefficients(dt, self.dispersion.get("debye", ()),
                                             self.dispersion.get("lorentz", ()), shp)
        eps = self.eps_r * EPS_0 + eps_add
        mu = self.mu_r * MU_0
        se = self.sigma_e * dt / (2.0 * eps)
        sm = self.sigma_m * dt / (2.0 * mu)
        self.ca = ((1.0 - se) / (1.0 + se)).astype(dtp)
        self.cb = ((dt / eps) / (1.0 + se)).astype(dtp)
        self.da = ((1.0 - sm) / (1.0 + sm)).astype(dtp)
        self.db = ((dt / mu) / (1.0 + sm)).astype(dtp)
        b, c = cpml_profile(n, self.dx, dt, self.R0, self.order) if n > 0 else (np.zeros(0), np.zeros(0))
        self.b, self.c = b.astype(dtp), c.astype(dtp)
        z = lambda *s: np.zeros(s, dtp)
        for f in ("ex", "ey", "ez", "hx", "hy", "hz"):
            setattr(self, f, z(B, nx, ny, nz))
        for nm in ("psi_hxy", "psi_hzy"):
            setattr(self, nm + "_lo", z(B, n, ny, nz)); setattr(self, nm + "_hi", z(B, n, ny, nz))
        for nm in ("psi_hyx", "psi_hzx"):
            setattr(self, nm + "_lo", z(B, nx, n, nz)); setattr(self, nm + "_hi", z(B, nx, n, nz))
        for nm in ("psi_hxz", "psi_hyz"):
            setattr(self, nm + "_lo", z(B, nx, ny, n)); setattr(self, nm + "_hi", z(B, nx, ny, n))
        self.deb = [tuple(a.astype(dtp) for a in t) for t in deb]
        self.lor = [tuple(a.astype(dtp) for a in t) for t in lor]
        self.j_deb = [z(3, B, nx, ny, nz) for _ in deb]
        self.j_lor = [z(3, B, nx, ny, nz) for _ in lor]
        self.j_lor_prev = [z(3, B, nx, ny, nz) for _ in lor]
        self.probe_data = np.zeros((B, len(self.prb), self.total_steps), dtp)
        self.step_index = 0

    def step(self):
        nx, ny, nz, n = self.nx, self.ny, self.nz, self.n
        t = self.dtype.type
        inv = t(1.0 / self.dx)
        ex, ey, ez, hx, hy, hz = self.ex, self.ey, self.ez, self.hx, self.hy, self.hz
        da, db, b, c = self.da[None], self.db[None], self.b, self.c
        A = slice(None)

        # interior H boxes (:764-818)
        s = (A, slice(n, nx - n), slice(n, ny - 1), slice(n, nz - 1))
        hx[s] = da[s] * hx[s] + db[s] * (
            (ey[A, n:nx - n, n:ny - 1, n + 1:nz] - ey[s]) * inv
            - (ez[A, n:nx - n, n + 1:ny, n:nz - 1] - ez[s]) * inv)
        s = (A, slice(n, nx - 1), slice(n, ny - n), slice(n, nz - 1))
        hy[s] = da[s] * hy[s] + db[s] * (
            (ez[A, n + 1:nx, n:ny - n, n:nz - 1] - ez[s]) * inv
            - (ex[A, n:nx - 1, n:ny - n, n + 1:nz] - ex[s]) * inv)
        s = (A, slice(n, nx - 1), slice(n, ny - 1), slice(n, nz - n))
        hz[s] = da[s] * hz[s] + db[s] * (
            (ex[A, n:nx - 1, n + 1:ny, n:nz - n] - ex[s]) * inv
            - (ey[A, n + 1:nx, n:ny - 1, n:nz - n] - ey[s]) * inv)

        if n > 0:
            self._cpml_h(inv)

        # interior E (:830-884); all three read the same (new) H
        I = (A, slice(n + 1, nx - n), slice(n + 1, ny - n), slice(n + 1, nz - n))
        xm = (A, slice(n, nx - n - 1), slice(n + 1, ny - n), slice(n + 1, nz - n))
        ym = (A, slice(n + 1, nx - n), slice(n, ny - n - 1), slice(n + 1, nz - n))
        zm = (A, slice(n + 1, nx - n), slice(n + 1, ny - n), slice(n, nz - n - 1))
        ca, cb = self.ca[None][I], self.cb[None][I]
        olds = (ex[I].copy(), ey[I].copy(), ez[I].copy())
        ex[I] = ca * ex[I] + cb * ((hz[I] - hz[ym]) * inv - (hy[I] - hy[zm]) * inv)
        ey[I] = ca * ey[I] + cb * ((hx[I] - hx[zm]) * inv - (hz[I] - hz[xm]) * inv)
        ez[I] = ca * ez[I] + cb * ((hy[I] - hy[xm]) * inv - (hx[I] - hx[ym]) * inv)
        if self.deb or self.lor:
            self._ade(I, cb, olds)

        # zero E on the low faces (:936-944), source and probes (:949-958)
        for f in (ex, ey, ez):
            f[:, 0, :, :] = 0
            f[:, :, 0, :] = 0
            f[:, :, :, 0] = 0
        st = self.step_index
        w = t(self.waveform[st])
        for bb, (sx, sy, sz) in enumerate(self.src):
            ez[bb, sx, sy, sz] += w
        for p, (px, py, pz) in enumerate(self.prb):
            self.probe_data[:, p, st] = ez[:, px, py, pz]
        self.step_index += 1

    def _cpml_h(self, inv):
        nx, ny, nz, n = self.nx, self.ny, self.nz, self.n
        ex, ey, ez, hx, hy, hz = self.ex, self.ey, self.ez, self.hx, self.hy, self.hz
        da, db = self.da[None], self.db[None]
        bl, cl = self.b, self.c
        br, cr = self.b[::-1], self.c[::-1]
        # x faces (:407-460): left uses forward, right backward differences
        B3 = lambda v: v[None, :, None, None]
        d = (ez[:, 1:n + 1] - ez[:, 0:n]) * inv
        self.psi_hxy_lo[:] = B3(bl) * self.psi_hxy_lo + B3(cl) * d
        hy[:, 0:n, :, :nz - 1] = da[:, 0:n, :, :nz - 1] * hy[:, 0:n, :, :nz - 1] - db[:, 0:n, :, :nz - 1] * self.psi_hxy_lo[:, :, :, :nz - 1]
        d = (ey[:, 1:n + 1] - ey[:, 0:n]) * inv
        self.psi_hzy_lo[:] = B3(bl) * self.psi_hzy_lo + B3(cl) * d
        hz[:, 0:n, :ny - 1, :] = da[:, 0:n, :ny - 1, :] * hz[:, 0:n, :ny - 1, :] + db[:, 0:n, :ny - 1, :] * self.psi_hzy_lo[:, :, :ny - 1, :]
        x0 = nx - n
        d = (ez[:, x0:nx] - ez[:, x0 - 1:nx - 1]) * inv
        self.psi_hxy_hi[:] = B3(br) * self.psi_hxy_hi + B3(cr) * d
        hy[:, x0:nx, :, :nz - 1] = da[:, x0:nx, :, :nz - 1] * hy[:, x0:nx, :, :nz - 1] - db[:, x0:nx, :, :nz - 1] * self.psi_hxy_hi[:, :, :, :nz - 1]
        d = (ey[:, x0:nx] - ey[:, x0 - 1:nx - 1]) * inv
        self.psi_hzy_hi[:] = B3(br) * self.psi_hzy_hi + B3(cr) * d
        hz[:, x0:nx, :ny - 1, :] = da[:, x0:nx, :ny - 1, :] * hz[:, x0:nx, :ny - 1, :] + db[:, x0:nx, :ny - 1, :] * self.psi_hzy_hi[:, :, :ny - 1, :]

        # y faces (:470-523)
        B3 = lambda v: v[None, None, :, None]
        d = (ez[:, :, 1:n + 1] - ez[:, :, 0:n]) * inv
        self.psi_hyx_lo[:] = B3(bl) * self.psi_hyx_lo + B3(cl) * d
        hx[:, :, 0:n, :nz - 1] = da[:, :, 0:n, :nz - 1] * hx[:, :, 0:n, :nz - 1] - db[:, :, 0:n, :nz - 1] * self.psi_hyx_lo[:, :, :, :nz - 1]
        d = (ex[:, :, 1:n + 1] - ex[:, :, 0:n]) * inv
        self.psi_hzx_lo[:] = B3(bl) * self.psi_hzx_lo + B3(cl) * d
        hz[:, :nx - 1, 0:n, :] = da[:, :nx - 1, 0:n, :] * hz[:, :nx - 1, 0:n, :] + db[:, :nx - 1, 0:n, :] * self.psi_hzx_lo[:, :nx - 1]
        y0 = ny - n
        d = (ez[:, :, y0:ny] - ez[:, :, y0 - 1:ny - 1]) * inv
        self.psi_hyx_hi[:] = B3(br) * self.psi_hyx_hi + B3(cr) * d
        hx[:, :, y0:ny, :nz - 1] = da[:, :, y0:ny, :nz - 1] * hx[:, :, y0:ny, :nz - 1] - db[:, :, y0:ny, :nz - 1] * self.psi_hyx_hi[:, :, :, :nz - 1]
        d = (ex[:, :, y0:ny] - ex[:, :, y0 - 1:ny - 1]) * inv
        self.psi_hzx_hi[:] = B3(br) * self.psi_hzx_hi + B3(cr) * d
        hz[:, :nx - 1, y0:ny, :] = da[:, :nx - 1, y0:ny, :] * hz[:, :nx - 1, y0:ny, :] + db[:, :nx - 1, y0:ny, :] * self.psi_hzx_hi[:, :nx - 1]

        # z faces (:533-586)
        B3 = lambda v: v[None, None, None, :]
        d = (ey[..., 1:n + 1] - ey[..., 0:n]) * inv
        self.psi_hxz_lo[:] = B3(bl) * self.psi_hxz_lo + B3(cl) * d
        hx[:, :, :ny - 1, 0:n] = da[:, :, :ny - 1, 0:n] * hx[:, :, :ny - 1, 0:n] + db[:, :, :ny - 1, 0:n] * self.psi_hxz_lo[:, :, :ny - 1]
        d = (ex[..., 1:n + 1] - ex[..., 0:n]) * inv
        self.psi_hyz_lo[:] = B3(bl) * self.psi_hyz_lo + B3(cl) * d
        hy[:, :nx - 1, :, 0:n] = da[:, :nx - 1, :, 0:n] * hy[:, :nx - 1, :, 0:n] - db[:, :nx - 1, :, 0:n] * self.psi_hyz_lo[:, :nx - 1]
        z0 = nz - n
        d = (ey[..., z0:nz] - ey[..., z0 - 1:nz - 1]) * inv
        self.psi_hxz_hi[:] = B3(br) * self.psi_hxz_hi + B3(cr) * d
        hx[:, :, :ny - 1, z0:nz] = da[:, :, :ny - 1, z0:nz] * hx[:, :, :ny - 1, z0:nz] + db[:, :, :ny - 1, z0:nz] * self.psi_hxz_hi[:, :, :ny - 1]
        d = (ex[..., z0:nz] - ex[..., z0 - 1:nz - 1]) * inv
        self.psi_hyz_hi[:] = B3(br) * self.psi_hyz_hi + B3(cr) * d
        hy[:, :nx - 1, :, z0:nz] = da[:, :nx - 1, :, z0:nz] * hy[:, :nx - 1, :, z0:nz] - db[:, :nx - 1, :, z0:nz] * self.psi_hyz_hi[:, :nx - 1]

    def _ade(self, I, cb, olds):
        """Debye/Lorentz currents on each E component inside the interior box,
        the 3D analogue of the 2D composition (dispersive.py:341-404,
        fdtd_2d.py:163-178): E -= cb*sum(gamma J), then the J recurrences."""
        sl = (slice(None),) + I[1:]
        dt = self.dtype.type(self.dt)
        for comp, f, old in zip(range(3), (self.ex, self.ey, self.ez), olds):
            sum_gj = 0.0
            for (k1, k2, g), J in zip(self.deb, self.j_deb):
                sum_gj = sum_gj + g[None][sl] * J[comp][I]
            for J in self.j_lor:
                sum_gj = sum_gj + J[comp][I]
            f[I] = f[I] - cb * sum_gj
            de_dt = (f[I] - old) / dt
            for (k1, k2, g), J in zip(self.deb, self.j_deb):
                J[comp][I] = k1[None][sl] * J[comp][I] + k2[None][sl] * de_dt
            for (k1, k2, k3), J, Jp in zip(self.lor, self.j_lor, self.j_lor_prev):
                j_new = k1[None][sl] * J[comp][I] + k3[None][sl] * Jp[comp][I] + k2[None][sl] * de_dt
                Jp[comp][I] = J[comp][I]
                J[comp][I] = j_new

    def run(self, steps=None):
        steps = self.total_steps - self.step_index if steps is None else steps
        for _ in range(steps):
            self.step()
        return self.probe_data

    def compute_energy(self):
        """fdtd_3d_batched.py:987-1011."""
        e = 0.5 * EPS_0 * float(np.sum(self.ex ** 2) + np.sum(self.ey ** 2) + np.sum(self.ez ** 2))
        h = 0.5 * MU_0 * float(np.sum(self.hx ** 2) + np.sum(self.hy ** 2) + np.sum(self.hz ** 2))
        return (e + h) * self.dx ** 3
