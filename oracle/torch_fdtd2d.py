"""PyTorch restatement of the batched 2D step for autograd — TEST INFRASTRUCTURE ONLY.

The reference's PyTorch backend cannot run its batched solver
(``torch.zeros(shape, dtype=np.float64)`` raises in src/ceep/core/backend.py:266-269),
so the gradient oracle is this functional restatement of the region map of
src/ceep/solvers/fdtd_2d_batched.py:454-526 (the same map as ``oracle.fdtd2d``,
to which it is pinned), with the Debye ADE composed as in
src/ceep/materials/dispersive.py:240-404.  Every update is written out of
place with masks so that ``torch.autograd`` differentiates the whole time
loop with respect to eps_r, sigma and the Debye delta_eps maps.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .fdtd2d import EPS_0, MU_0, cpml_profile, gaussian_derivative_waveform, reference_dt_2d


def coefficients(eps_r, sigma, debye, dt, lorentz=()):
    """ca, cb, dt/(eps_r eps0) and per-pole coefficients as differentiable
    tensors: Debye (k1, k2, gamma), then Lorentz (k1, k2, k3)
    (dispersive.py:253-261, :278-299)."""
    eps = eps_r * EPS_0
    poles = []
    for de, tau in debye:
        valid = tau > 0
        den = 2.0 * tau + dt
        k1 = torch.where(valid, (2.0 * tau - dt) / den, torch.zeros_like(tau))
        k2 = torch.where(valid, 2.0 * EPS_0 * de * dt / den, torch.zeros_like(tau))
        g = torch.where(valid, (1.0 + k1) / 2.0, torch.zeros_like(tau))
        eps = eps + k2 / 2.0
        poles.append((k1, k2, g))
    for de, w0, dl in lorentz:
        valid = w0 > 0
        w02, dt2 = w0 * w0, dt * dt
        den = 4.0 + 2.0 * dl * dt + w02 * dt2
        z = torch.zeros_like(w0)
        k1 = torch.where(valid, (8.0 - 2.0 * w02 * dt2) / den, z)
        k3 = torch.where(valid, -(4.0 - 2.0 * dl * dt + w02 * dt2) / den, z)
        k2 = torch.where(valid, 2.0 * EPS_0 * de * w02 * dt2 / den, z)
        eps = eps + k2 / 2.0
        poles.append((k1, k2, k3))
    s = sigma * dt / (2.0 * eps)
    ca = (1.0 - s) / (1.0 + s)
    cb = (dt / eps) / (1.0 + s)
    dteps = dt / (eps_r * EPS_0)
    return ca, cb, dteps, poles


class TorchFdtd2D:
    """Batched 2D TMz with autograd; state (B, nx, ny) float64."""

    def __init__(self, nx, ny, dx, total_steps, cpml_thickness, source_positions, probe_positions,
                 frequency, delay_factor=5.0, device="cpu"):
        self.nx, self.ny, self.dx, self.T, self.n = nx, ny, dx, total_steps, cpml_thickness
        self.src, self.prb = list(source_positions), list(probe_positions)
        self.B = len(self.src)
        self.dt = reference_dt_2d(dx)
        self.device = torch.device(device)
        self.w = torch.as_tensor(gaussian_derivative_waveform(total_steps, self.dt, frequency, delay_factor),
                                 dtype=torch.float64, device=self.device)
        self._masks()

    def _masks(self):
        nx, ny, n = self.nx, self.ny, self.n
        x = np.arange(nx)[:, None] * np.ones((1, ny), int)
        y = np.ones((nx, 1), int) * np.arange(ny)[None, :]
        b, c = cpml_profile(n, self.dx, self.dt) if n > 0 else (np.zeros(1), np.zeros(1))
        t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=self.device)
        self.F7x = t((x >= n) & (x < nx - n) & (y >= n) & (y < ny - 1))
        self.F7y = t((x >= n) & (x < nx - 1) & (y >= n) & (y < ny - n))
        self.F9 = t((x >= n + 1) & (x < nx - n) & (y >= n + 1) & (y < ny - n))
        self.F9b = self.F9 > 0
        # H strips and their coefficient index
        sy = (y < n) | ((y >= ny - n) & (y < ny - 1))
        iy = np.where(y < n, y, ny - 1 - y).clip(0, max(n - 1, 0))
        sx = (x < n) | ((x >= nx - n) & (x < nx - 1))
        ix = np.where(x < n, x, nx - 1 - x).clip(0, max(n - 1, 0))
        # E strips
        sex = (y >= 1) & (((x >= 1) & (x <= n)) | (x >= nx - n)) & (n > 0)
        iex = np.where((x >= 1) & (x <= n), x - 1, nx - 1 - x).clip(0, max(n - 1, 0))
        sey = (x >= 1) & (((y >= 1) & (y <= n)) | (y >= ny - n)) & (n > 0)
        iey = np.where((y >= 1) & (y <= n), y - 1, ny - 1 - y).clip(0, max(n - 1, 0))
        self.Sy, self.Sx, self.SEx, self.SEy = t(sy & (n > 0)), t(sx & (n > 0)), t(sex), t(sey)
        self.by, self.cy = t(b[iy]), t(c[iy])
        self.bx, self.cx = t(b[ix]), t(c[ix])
        self.bex, self.cex = t(b[iex]), t(c[iex])
        self.bey, self.cey = t(b[iey]), t(c[iey])
        self.notedge = t(~((x == 0) | (x == nx - 1) | (y == 0) | (y == ny - 1)))
        src = np.zeros((self.B, nx, ny))
        for k, (sx_, sy_) in enumerate(self.src):
            src[k, sx_, sy_] = 1.0
        self.srcmask = t(src)

    def run(self, eps_r, sigma, debye=(), lorentz=()):
        """Probe series (B, P, T) as a differentiable function of the maps
        (Debye poles (delta_eps, tau), Lorentz poles (delta_eps, omega_0, delta))."""
        dt, inv = self.dt, 1.0 / self.dx
        db = dt / MU_0
        dbdx = db * inv
        ca, cb, dteps, poles = coefficients(eps_r, sigma, debye, dt, lorentz)
        nd = len(debye)
        B, nx, ny = self.B, self.nx, self.ny
        z = torch.zeros((B, nx, ny), dtype=torch.float64, device=self.device)
        E, X, Y, PHX, PHY, PEX, PEY = z, z, z, z, z, z, z
        J = [z for _ in poles]
        Jp = [z for _ in poles[nd:]]
        px = torch.as_tensor([p[0] for p in self.prb], device=self.device)
        py = torch.as_tensor([p[1] for p in self.prb], device=self.device)
        out = []
        for st in range(self.T):
            dEx = torch.nn.functional.pad(E[:, 1:, :] - E[:, :-1, :], (0, 0, 0, 1))
            dEy = torch.nn.functional.pad(E[:, :, 1:] - E[:, :, :-1], (0, 1))
            X1 = X - dbdx * self.F7x * dEy
            PHX1 = torch.where(self.Sy > 0, self.by * PHX + self.cy * (dEy * inv), PHX)
            X1 = X1 - db * self.Sy * PHX1
            Y1 = Y + dbdx * self.F7y * dEx
            PHY1 = torch.where(self.Sx > 0, self.bx * PHY + self.cx * (dEx * inv), PHY)
            Y1 = Y1 + db * self.Sx * PHY1
            cY = Y1 - torch.nn.functional.pad(Y1[:, :-1, :], (0, 0, 1, 0))
            cX = X1 - torch.nn.functional.pad(X1[:, :, :-1], (1, 0))
            e1 = ca * E + cb * (cY * inv - cX * inv)
            if poles:
                # Debye J carries gamma, Lorentz J enters with gamma = 1
                sgj = sum(c[2] * j if q < nd else j for q, (c, j) in enumerate(zip(poles, J)))
                e1 = e1 - cb * sgj
                dedt = (e1 - E) / dt
                newJ = [torch.where(self.F9b, k1 * j + k2 * dedt, j) for (k1, k2, g), j in zip(poles[:nd], J[:nd])]
                newJ += [torch.where(self.F9b, k1 * j + k3 * jp + k2 * dedt, j)
                         for (k1, k2, k3), j, jp in zip(poles[nd:], J[nd:], Jp)]
                Jp = [torch.where(self.F9b, j, jp) for j, jp in zip(J[nd:], Jp)]
                J = newJ
            E1 = torch.where(self.F9b, e1, E)
            PEX = torch.where(self.SEx > 0, self.bex * PEX + self.cex * (cY * inv), PEX)
            E2 = E1 + self.SEx * dteps * PEX
            PEY = torch.where(self.SEy > 0, self.bey * PEY + self.cey * (cX * inv), PEY)
            E3 = E2 - self.SEy * dteps * PEY
            E = E3 * self.notedge + self.w[st] * self.srcmask
            X, Y, PHX, PHY = X1, Y1, PHX1, PHY1
            out.append(E[:, px, py])
        return torch.stack(out, dim=-1)


def s_misfit_loss(probes, dt, frequencies, target):
    """L = sum |S - S*|^2 with S[f, rx, tx] the running DFT (dft.py:55-90)."""
    T = probes.shape[-1]
    w = 2.0 * math.pi * torch.as_tensor(frequencies, dtype=torch.float64, device=probes.device)
    ph = w[:, None] * (torch.arange(T, dtype=torch.float64, device=probes.device) * dt)[None, :]
    tw = torch.complex(torch.cos(ph) * dt, -torch.sin(ph) * dt)            # (F, T)
    S = torch.einsum("bpt,ft->fpb", probes.to(torch.complex128), tw)
    return (S - target).abs().pow(2).sum(), S
