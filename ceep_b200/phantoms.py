"""Seeded synthetic head phantoms for the batched 2D path.

``HeadPhantom2D`` generalises the layer geometry of the reference's
``BrainPhantom2D`` (src/ceep/phantoms/head_models.py:497-631: skin 3 mm,
skull 7 mm, CSF 2 mm, grey matter 10 mm, white matter inside; outside-in
assignment) from circles to ellipses with seeded +/-5 % jitter, and gives each
layer one Debye pole drawn from seeded uniform ranges.  A seeded disk
(haemorrhage) is added with probability ``p_disk``.  It satisfies the
``set_phantom`` duck typing (``get_eps_map``) and adds ``get_dispersion``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

LAYERS = ("skin", "skull", "csf", "grey", "white")
THICKNESS = (3e-3, 7e-3, 2e-3, 10e-3)  # skin, skull, csf, grey (head_models.py:541-545)


@dataclass
class HeadPhantom2D:
    nx: int = 600
    ny: int = 600
    dx: float = 0.5e-3
    seed: int = 0
    semi_axes: tuple = (0.09, 0.07)          # metres
    jitter: float = 0.05
    eps_inf: tuple = (4.0, 40.0)
    delta_eps: tuple = (10.0, 45.0)
    tau: tuple = (5e-12, 15e-12)
    sigma: tuple = (0.1, 2.5)
    disk_radius: tuple = (0.6e-2, 1.5e-2)
    disk_eps: tuple = (55.0, 65.0)
    disk_sigma: tuple = (1.4, 1.8)
    p_disk: float = 0.8
    layer_params: dict = field(init=False)

    def __post_init__(self):
        rng = np.random.default_rng(self.seed)
        u = lambda r: float(rng.uniform(*r))
        self.a = self.semi_axes[0] * (1 + rng.uniform(-self.jitter, self.jitter))
        self.b = self.semi_axes[1] * (1 + rng.uniform(-self.jitter, self.jitter))
        self.layer_params = {name: dict(eps_inf=u(self.eps_inf), delta_eps=u(self.delta_eps), tau=u(self.tau),
                                         sigma=u(self.sigma)) for name in LAYERS}
        self.has_disk = bool(rng.random() < self.p_disk)
        if self.has_disk:
            r = u(self.disk_radius)
            # centre inside the white-matter ellipse, fully contained
            inner_a = self.a - sum(THICKNESS) - r
            inner_b = self.b - sum(THICKNESS) - r
            ang, rad = rng.uniform(0, 2 * np.pi), np.sqrt(rng.uniform(0, 1)) * 0.8
            self.disk = dict(cx=rad * inner_a * np.cos(ang), cy=rad * inner_b * np.sin(ang), r=r,
                             eps=u(self.disk_eps), sigma=u(self.disk_sigma))
        else:
            self.disk = None
        self._maps = None

    def _build(self):
        if self._maps is not None:
            return self._maps
        nx, ny, dx = self.nx, self.ny, self.dx
        x, y = np.meshgrid((np.arange(nx) - nx // 2) * dx, (np.arange(ny) - ny // 2) * dx, indexing="ij")
        eps = np.ones((nx, ny))
        sig = np.zeros((nx, ny))
        de = np.zeros((nx, ny))
        tau = np.zeros((nx, ny))
        shrink = 0.0
        for k, name in enumerate(LAYERS):
            a, b = self.a - shrink, self.b - shrink
            m = (x / a) ** 2 + (y / b) ** 2 <= 1.0
            p = self.layer_params[name]
            eps[m], sig[m], de[m], tau[m] = p["eps_inf"], p["sigma"], p["delta_eps"], p["tau"]
            if k < len(THICKNESS):
                shrink += THICKNESS[k]
        if self.disk is not None:
            d = self.disk
            m = (x - d["cx"]) ** 2 + (y - d["cy"]) ** 2 <= d["r"] ** 2
            eps[m], sig[m], de[m], tau[m] = d["eps"], d["sigma"], 0.0, 0.0
        self._maps = (eps, sig, de, tau)
        return self._maps

    def get_eps_map(self, frequency: float = 0.0):
        """(eps_inf, sigma) maps; eps_r of the solver holds eps_inf for Debye cells."""
        eps, sig, _, _ = self._build()
        return eps.copy(), sig.copy()

    def get_dispersion(self):
        _, _, de, tau = self._build()
        return {"debye": [(de.copy(), tau.copy())], "lorentz": []}


@dataclass
class LorentzHeadPhantom2D(HeadPhantom2D):
    """Same geometry with a two-pole Lorentz model per layer in place of Debye
    (omega_0 / 2 pi in [1, 20] GHz, delta / 2 pi in [0.1, 1] GHz)."""
    f0: tuple = (1e9, 20e9)
    fdamp: tuple = (0.1e9, 1e9)
    lorentz_delta_eps: tuple = (1.0, 10.0)

    def __post_init__(self):
        super().__post_init__()
        rng = np.random.default_rng(self.seed + 7919)
        self.lorentz_params = {name: [dict(delta_eps=float(rng.uniform(*self.lorentz_delta_eps)),
                                           w0=2 * np.pi * float(rng.uniform(*self.f0)),
                                           d=2 * np.pi * float(rng.uniform(*self.fdamp))) for _ in range(2)]
                               for name in LAYERS}

    def get_dispersion(self):
        eps, _, de, _ = self._build()
        nx, ny = self.nx, self.ny
        poles = [(np.zeros((nx, ny)), np.zeros((nx, ny)), np.zeros((nx, ny))) for _ in range(2)]
        # layer membership is recovered from the Debye delta_eps map, which is unique per layer
        for name in LAYERS:
            m = de == self.layer_params[name]["delta_eps"]
            for q in range(2):
                lp = self.lorentz_params[name][q]
                poles[q][0][m], poles[q][1][m], poles[q][2][m] = lp["delta_eps"], lp["w0"], lp["d"]
        return {"debye": [], "lorentz": poles}


def ring_positions(n_ant: int, center: tuple, radius: float):
    """Antenna grid positions of the dataset generator's circle
    (scripts/generate_corrected_dataset.py:121-129): angles from
    np.linspace(0, 2 pi, n, endpoint=False), radius in cells, int()
    truncation."""
    ang = np.linspace(0, 2 * np.pi, n_ant, endpoint=False)
    return [(int(center[0] + radius * np.cos(a)), int(center[1] + radius * np.sin(a))) for a in ang]


def circular_array_positions(num_antennas: int, radius_mm: float, center: tuple, dx: float):
    """Antenna grid positions of ``CircularArray`` (src/ceep/antennas/arrays.py:
    110-143): angle 2 pi i / n, offset radius_m cos(angle) / dx (radius in
    metres), int() truncation; a third centre coordinate is carried through.
    The angle and the division by dx are formed as there, so the truncation
    lands on the same cell (ring_positions can differ by one cell where
    r cos(angle) is within an ulp of an integer)."""
    radius = radius_mm * 1e-3
    out = []
    for i in range(num_antennas):
        angle = 2 * np.pi * i / num_antennas
        x_off = radius * np.cos(angle) / dx
        y_off = radius * np.sin(angle) / dx
        pos = (int(center[0] + x_off), int(center[1] + y_off))
        out.append(pos + ((int(center[2]),) if len(center) == 3 else ()))
    return out


@dataclass
class HeadPhantom3D:
    """Concentric ellipsoid shells (the 2D layer sequence, thicknesses from
    head_models.py:541-545) with one seeded Debye pole per shell and a seeded
    ellipsoidal inclusion of 0.8-1.5 cm; ``get_eps_map_3d`` feeds
    ``BatchedFDTD3D.set_phantom``.  ``with_inclusion=False`` gives the same
    head without the inclusion (the same draws, so the shells are identical)."""
    nx: int = 192
    ny: int = 192
    nz: int = 192
    dx: float = 1e-3
    seed: int = 0
    semi_axes: tuple = (0.070, 0.056, 0.060)
    jitter: float = 0.05
    eps_inf: tuple = (4.0, 40.0)
    delta_eps: tuple = (10.0, 45.0)
    tau: tuple = (5e-12, 15e-12)
    sigma: tuple = (0.1, 2.5)
    inclusion_radius: tuple = (0.8e-2, 1.5e-2)
    inclusion_eps: tuple = (55.0, 65.0)
    inclusion_sigma: tuple = (1.4, 1.8)
    with_inclusion: bool = True

    def __post_init__(self):
        rng = np.random.default_rng(self.seed)
        u = lambda r: float(rng.uniform(*r))
        self.axes = tuple(a * (1 + rng.uniform(-self.jitter, self.jitter)) for a in self.semi_axes)
        self.layer_params = {name: dict(eps_inf=u(self.eps_inf), delta_eps=u(self.delta_eps), tau=u(self.tau),
                                         sigma=u(self.sigma)) for name in LAYERS}
        r = u(self.inclusion_radius)
        radii = (r, r * rng.uniform(0.7, 1.0), r * rng.uniform(0.7, 1.0))
        inner = [a - sum(THICKNESS) - r for a in self.axes]
        c = [rng.uniform(-0.6, 0.6) * max(v, 0.0) for v in inner]
        self.inclusion = dict(center=c, radii=radii, eps=u(self.inclusion_eps), sigma=u(self.inclusion_sigma))
        self._maps = None

    def _build(self):
        if self._maps is not None:
            return self._maps
        g = lambda n: (np.arange(n) - n // 2) * self.dx
        x, y, z = np.meshgrid(g(self.nx), g(self.ny), g(self.nz), indexing="ij")
        eps, sig = np.ones(x.shape), np.zeros(x.shape)
        de, tau = np.zeros(x.shape), np.zeros(x.shape)
        shrink = 0.0
        for k, name in enumerate(LAYERS):
            a, b, c = (v - shrink for v in self.axes)
            m = (x / a) ** 2 + (y / b) ** 2 + (z / c) ** 2 <= 1.0
            p = self.layer_params[name]
            eps[m], sig[m], de[m], tau[m] = p["eps_inf"], p["sigma"], p["delta_eps"], p["tau"]
            if k < len(THICKNESS):
                shrink += THICKNESS[k]
        inc = self.inclusion
        (cx, cy, cz), (rx, ry, rz) = inc["center"], inc["radii"]
        m = ((x - cx) / rx) ** 2 + ((y - cy) / ry) ** 2 + ((z - cz) / rz) ** 2 <= 1.0
        if self.with_inclusion:
            eps[m], sig[m], de[m], tau[m] = inc["eps"], inc["sigma"], 0.0, 0.0
        self._maps = (eps, sig, de, tau)
        return self._maps

    def get_eps_map_3d(self, frequency: float = 0.0):
        eps, sig, _, _ = self._build()
        return eps.copy(), sig.copy()

    def get_dispersion(self):
        _, _, de, tau = self._build()
        return {"debye": [(de.copy(), tau.copy())], "lorentz": []}
