"""PyTorch restatement of the batched 3D step for autograd — TEST INFRASTRUCTURE ONLY.

Functional (out-of-place, masked) restatement of the probe series of
src/ceep/solvers/fdtd_3d_batched.py:886-985 (the map of ``oracle.fdtd3d``, to
which it is pinned) with the Debye ADE on each E component, so that
``torch.autograd`` differentiates the whole time loop with respect to eps_r,
sigma and the Debye delta_eps / tau maps.

The H-CPML face updates (:398-586) are left out because they cannot change a
probe value: E is updated only on [n+1, N-n)^3 (:820-884); there it reads H
on [n, N-n)^3, where no cell lies on a CPML face; those H cells take only the
plain box update (:753-818), which reads E on [n, N-n]^3, i.e. interior E or
E cells the step never changes (zeroed on the low faces, plus the source).
So E everywhere, and with it every probe, is the same with or without the
faces.  ``tests/test_adjoint3d_cpu.py`` checks this against the full oracle.
mu_r = 1 and sigma_m = 0 (da = 1, db = dt/mu0), as in the reference's defaults.
"""
from __future__ import annotations

import numpy as np
import torch

from .fdtd2d import MU_0, gaussian_derivative_waveform
from .fdtd3d import reference_dt_3d
from .torch_fdtd2d import coefficients

_pad = torch.nn.functional.pad


def _fwd(f, axis):
    """f[i+1] - f[i] along `axis` (1, 2, 3 of (B, nx, ny, nz)), 0 at the last index."""
    d = f.narrow(axis, 1, f.shape[axis] - 1) - f.narrow(axis, 0, f.shape[axis] - 1)
    pad = [0, 0] * (3 - axis) + [0, 1]
    return _pad(d, pad)


def _bwd(f, axis):
    """f[i] - f[i-1] along `axis`, with f[-1] = 0."""
    pad = [0, 0] * (3 - axis) + [1, 0]
    return f - _pad(f.narrow(axis, 0, f.shape[axis] - 1), pad)


class TorchFdtd3D:
    """Batched 3D Yee FDTD with autograd; state (B, nx, ny, nz) float64."""

    def __init__(self, nx, ny, nz, dx, total_steps, cpml_thickness, source_positions, probe_positions,
                 frequency, delay_factor=5.0, device="cpu"):
        self.nx, self.ny, self.nz, self.dx = nx, ny, nz, dx
        self.T, self.n = total_steps, cpml_thickness
        self.src, self.prb = list(source_positions), list(probe_positions)
        self.B = len(self.src)
        self.dt = reference_dt_3d(dx)
        self.device = torch.device(device)
        self.w = torch.as_tensor(gaussian_derivative_waveform(total_steps, self.dt, frequency, delay_factor),
                                 dtype=torch.float64, device=self.device)
        x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        n = self.n
        t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=self.device)
        rng = lambda v, lo, hi: (v >= lo) & (v < hi)
        self.box_x = t(rng(x, n, nx - n) & rng(y, n, ny - 1) & rng(z, n, nz - 1))
        self.box_y = t(rng(x, n, nx - 1) & rng(y, n, ny - n) & rng(z, n, nz - 1))
        self.box_z = t(rng(x, n, nx - 1) & rng(y, n, ny - 1) & rng(z, n, nz - n))
        self.inner = torch.as_tensor(rng(x, n + 1, nx - n) & rng(y, n + 1, ny - n) & rng(z, n + 1, nz - n),
                                     device=self.device)
        self.notlow = t(~((x == 0) | (y == 0) | (z == 0)))
        src = np.zeros((self.B, nx, ny, nz))
        for k, (a, b, c) in enumerate(self.src):
            src[k, a, b, c] = 1.0
        self.srcmask = t(src)

    def run(self, eps_r, sigma, debye=()):
        """Probe series (B, P, T) of Ez as a differentiable function of the maps."""
        dt, inv = self.dt, 1.0 / self.dx
        dbi = dt / MU_0 * inv
        ca, cb, _, poles = coefficients(eps_r, sigma, debye, dt)
        z = torch.zeros((self.B, self.nx, self.ny, self.nz), dtype=torch.float64, device=self.device)
        Ex, Ey, Ez, Hx, Hy, Hz = z, z, z, z, z, z
        J = [[z, z, z] for _ in poles]
        P = [torch.as_tensor([p[i] for p in self.prb], device=self.device) for i in range(3)]
        out = []
        for st in range(self.T):
            Hx = Hx + self.box_x * dbi * (_fwd(Ey, 3) - _fwd(Ez, 2))
            Hy = Hy + self.box_y * dbi * (_fwd(Ez, 1) - _fwd(Ex, 3))
            Hz = Hz + self.box_z * dbi * (_fwd(Ex, 2) - _fwd(Ey, 1))
            curls = ((_bwd(Hz, 2) - _bwd(Hy, 3)) * inv, (_bwd(Hx, 3) - _bwd(Hz, 1)) * inv,
                     (_bwd(Hy, 1) - _bwd(Hx, 2)) * inv)
            new = []
            for c, (E, cu) in enumerate(zip((Ex, Ey, Ez), curls)):
                e = ca * E + cb * cu
                if poles:
                    e = e - cb * sum(g * j[c] for (k1, k2, g), j in zip(poles, J))
                    dedt = (e - E) / dt
                    for (k1, k2, g), j in zip(poles, J):
                        j[c] = torch.where(self.inner, k1 * j[c] + k2 * dedt, j[c])
                new.append(torch.where(self.inner, e, E) * self.notlow)
            Ex, Ey, Ez = new[0], new[1], new[2] + self.w[st] * self.srcmask
            out.append(Ez[:, P[0], P[1], P[2]])
        return torch.stack(out, dim=-1)
