"""Drop-in for the reference's non-batched 2D solver family, on the B200.

Mirrors, with the reference's names and semantics:

* ``SimulationMode``, ``GridConfig``, ``SimulationConfig``  (src/ceep/core/config.py:24-215)
* ``Grid2D`` material maps and coefficients              (src/ceep/core/grid.py:51-344)
* ``GaussianSource``, ``SinusoidalSource``,
  ``ModulatedGaussianSource``                             (src/ceep/sources/waveforms.py:25-130)
* ``PEC``, ``MurABC``, ``CPML`` (CFS-CPML)                (src/ceep/boundaries/absorbing.py:48-561)
* ``DFTMonitor``                                          (src/ceep/solvers/dft.py:16-120)
* ``FDTD2D`` (TMz and TEz)                                 (src/ceep/solvers/fdtd_2d.py:42-344,
                                                           src/ceep/solvers/fdtd_base.py:30-218)

The time loop runs in ``libceep_b200.so`` (``ceep2s_*``, ``csrc/single2d.cu``):
per step an H kernel (update + CPML H), an E kernel (update, E sources,
boundary operations in list order), and small epilogues (TEz Hz sources,
Mur edges, probe / monitor recording, snapshots), the whole ``run()``
captured into one CUDA graph.  Fields are FP32 device tensors in the
reference's (nx, ny) layout; materials and update coefficients are computed
on the host in FP64 as the reference does and rounded once.

The solver also accepts the reference's own config, source and boundary
objects (duck typing: ``config.grid.nx/ny/dx/dy``, ``config.dt``,
``config.mode.name``, ``config.num_steps``; sources with ``position``,
``component`` and ``value_at``; boundaries by class name).

Divergences, by design: snapshots are copies (on the NumPy array module the
reference's snapshots alias the live field, so they all show the last
step); ``dft_monitors`` work (the reference's FDTD2D calls a
``DFTMonitor.initialize`` that does not exist); a source on a component the
mode lacks raises ``ValueError`` up front where the reference raises
IndexError mid-run; MurABC must be the last boundary and one CPML at most;
dispersive (Debye) materials in this solver are not supported
(``NotImplementedError``).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from enum import Enum, auto
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from ._lib import check, lib
from .constants import C_0, EPS_0, MU_0, cfl_timestep_2d, cfl_timestep_3d
from .physics import rdiv

TWO_PI = 2.0 * math.pi


# -- configuration (config.py) -------------------------------------------------------
class SimulationMode(Enum):
    TMZ = auto()
    TEZ = auto()
    FULL_3D = auto()


@dataclass
class GridConfig:
    nx: int
    ny: int
    nz: int = 1
    dx: float = 1e-3
    dy: float = 1e-3
    dz: float = 1e-3

    def __post_init__(self) -> None:
        if self.nx <= 0 or self.ny <= 0 or self.nz <= 0:
            raise ValueError("Grid dimensions must be positive integers.")
        if self.dx <= 0 or self.dy <= 0 or self.dz <= 0:
            raise ValueError("Grid spacings must be positive.")

    @property
    def is_3d(self) -> bool:
        return self.nz > 1

    @property
    def shape(self) -> Tuple[int, ...]:
        return (self.nx, self.ny, self.nz) if self.is_3d else (self.nx, self.ny)

    @property
    def total_cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def physical_size(self) -> Tuple[float, ...]:
        if self.is_3d:
            return (self.nx * self.dx, self.ny * self.dy, self.nz * self.dz)
        return (self.nx * self.dx, self.ny * self.dy)


@dataclass
class SimulationConfig:
    grid: GridConfig
    mode: SimulationMode = SimulationMode.TMZ
    courant: float = 0.5
    total_time: Optional[float] = None
    total_steps: Optional[int] = None
    backend: Optional[object] = None

    def __post_init__(self) -> None:
        max_courant = 1.0 / math.sqrt(3.0 if self.grid.is_3d else 2.0)
        if self.courant <= 0 or self.courant > max_courant:
            raise ValueError(f"Courant number must be in (0, {max_courant:.4f}] for "
                             f"{'3D' if self.grid.is_3d else '2D'} simulation. Got {self.courant}.")
        if self.total_time is None and self.total_steps is None:
            raise ValueError("Must specify either total_time or total_steps.")

    @property
    def dt(self) -> float:
        g = self.grid
        if g.is_3d:
            return cfl_timestep_3d(g.dx, g.dy, g.dz, self.courant)
        return cfl_timestep_2d(g.dx, g.dy, self.courant)

    @property
    def num_steps(self) -> int:
        if self.total_steps is not None:
            return self.total_steps
        return int(math.ceil(self.total_time / self.dt))


# -- sources (waveforms.py) ---------------------------------------------------------
@dataclass
class GaussianSource:
    """A exp(-((t - t0)/tau)^2), tau = 1/(pi f_max), t0 = delay_factor tau."""
    x: int
    y: int
    frequency_max: float
    amplitude: float = 1.0
    delay_factor: float = 6.0
    field_component: str = "Ez"
    z: int = 0

    def __post_init__(self) -> None:
        self._tau = 1.0 / (math.pi * self.frequency_max)
        self._t0 = self.delay_factor * self._tau

    def value_at(self, timestep: int, dt: float) -> float:
        t = timestep * dt
        return self.amplitude * math.exp(-((t - self._t0) / self._tau) ** 2)

    position = property(lambda self: (self.x, self.y))
    component = property(lambda self: self.field_component)
    tau = property(lambda self: self._tau)
    t0 = property(lambda self: self._t0)

    def waveform(self, num_steps: int, dt: float) -> np.ndarray:
        t = np.arange(num_steps) * dt
        return self.amplitude * np.exp(-((t - self._t0) / self._tau) ** 2)


@dataclass
class SinusoidalSource:
    """A sin(2 pi f t) with the ramp 1 - exp(-(t / 2T)^2)."""
    x: int
    y: int
    frequency: float
    amplitude: float = 1.0
    field_component: str = "Ez"
    z: int = 0

    def value_at(self, timestep: int, dt: float) -> float:
        t = timestep * dt
        period = 1.0 / self.frequency
        ramp = 1.0 - math.exp(-((t / (2.0 * period)) ** 2))
        return self.amplitude * math.sin(TWO_PI * self.frequency * t) * ramp

    position = property(lambda self: (self.x, self.y))
    component = property(lambda self: self.field_component)

    def waveform(self, num_steps: int, dt: float) -> np.ndarray:
        t = np.arange(num_steps) * dt
        period = 1.0 / self.frequency
        ramp = 1.0 - np.exp(-((t / (2.0 * period)) ** 2))
        return self.amplitude * np.sin(TWO_PI * self.frequency * t) * ramp


@dataclass
class ModulatedGaussianSource:
    """A exp(-((t - t0)/tau)^2) sin(2 pi f t), tau = 1/(pi bandwidth)."""
    x: int
    y: int
    frequency: float
    bandwidth: float
    amplitude: float = 1.0
    delay_factor: float = 6.0
    field_component: str = "Ez"
    z: int = 0

    def __post_init__(self) -> None:
        self._tau = 1.0 / (math.pi * self.bandwidth)
        self._t0 = self.delay_factor * self._tau

    def value_at(self, timestep: int, dt: float) -> float:
        t = timestep * dt
        envelope = math.exp(-((t - self._t0) / self._tau) ** 2)
        return self.amplitude * envelope * math.sin(TWO_PI * self.frequency * t)

    position = property(lambda self: (self.x, self.y))
    component = property(lambda self: self.field_component)

    def waveform(self, num_steps: int, dt: float) -> np.ndarray:
        t = np.arange(num_steps) * dt
        return self.amplitude * np.exp(-((t - self._t0) / self._tau) ** 2) * np.sin(TWO_PI * self.frequency * t)


# -- boundaries (absorbing.py) ------------------------------------------------------
@dataclass
class PEC:
    """Tangential E zeroed on the four edges after each E update."""


@dataclass
class MurABC:
    """First-order Mur on the edges of Ez (TMz) or Hz (TEz)."""


@dataclass
class CPML:
    """CFS-CPML: sigma = sigma_max rho^order, kappa = 1 + (kappa_max - 1) rho^order,
    alpha = alpha_max (1 - rho), sigma_max = sigma_factor (order + 1) / (150 pi d)."""
    thickness: int = 10
    order: int = 4
    sigma_factor: float = 2.0
    alpha_max: float = 0.05
    kappa_max: float = 1.0


def cpml_coefficients(n: int, d: float, dt: float, order, sigma_factor, alpha_max, kappa_max):
    """be, ce (E positions rho = k/n) and bh, ch (H positions rho = (k + 1/2)/n),
    FP64 (absorbing.py:262-300)."""
    sigma_max = sigma_factor * (order + 1) / (150.0 * math.pi * d)
    out = []
    for half in (0.0, 0.5):
        rho = (np.arange(n, dtype=np.float64) + half) / n
        sig = sigma_max * rho ** order
        kap = 1.0 + (kappa_max - 1.0) * rho ** order
        alp = alpha_max * (1.0 - rho)
        b = np.exp(-(sig / kap + alp) * dt / EPS_0)
        c = np.where(np.abs(sig) < 1e-20, 0.0, sig / (sig * kap + kap ** 2 * alp) * (b - 1.0))
        out += [b, c]
    return out


# -- DFT monitor (dft.py) -------------------------------------------------------------
class DFTMonitor:
    """Running DFT sum_n F(n dt) e^{-j w n dt} dt of a field region."""

    def __init__(self, frequencies, region, component: str = "Ez"):
        self.frequencies = np.atleast_1d(frequencies).astype(np.float64)
        self.region = region
        self.component = component
        self.omega = 2.0 * np.pi * self.frequencies
        self.dft_real = None
        self.dft_imag = None
        self._initialized = False

    def _initialize(self, shape) -> None:
        nf = len(self.frequencies)
        self.dft_real = np.zeros((nf,) + tuple(shape))
        self.dft_imag = np.zeros((nf,) + tuple(shape))
        self._initialized = True

    def update(self, field, step: int, dt: float) -> None:
        """One step on a host array, as the reference's update (dft.py:52-90)."""
        region = np.asarray(field)[self.region]
        if not self._initialized:
            self._initialize(np.shape(region))
        t = step * dt
        shp = [len(self.frequencies)] + [1] * np.ndim(region)
        self.dft_real += np.cos(self.omega * t).reshape(shp) * region * dt
        self.dft_imag += (-np.sin(self.omega * t)).reshape(shp) * region * dt

    def get_complex_field(self) -> np.ndarray:
        if not self._initialized:
            raise RuntimeError("Monitor has not received any updates yet.")
        return self.dft_real + 1j * self.dft_imag


# -- grid (grid.py) -------------------------------------------------------------------
_FIELDS = {"TMZ": ("ez", "hx", "hy"), "TEZ": ("hz", "ex", "ey")}
_COMP = {"TMZ": {"Ez": 0, "Hx": 1, "Hy": 2}, "TEZ": {"Hz": 0, "Ex": 1, "Ey": 2}}


def _mode_name(config) -> str:
    m = config.mode
    return getattr(m, "name", str(m)).upper()


class Grid2D:
    """Yee grid of one 2D simulation: FP32 device fields in the reference's
    (nx, ny) layout, FP64 host material maps and update coefficients."""

    def __init__(self, config, device="cuda"):
        self.config = config
        mode = _mode_name(config)
        if mode not in _FIELDS:
            raise ValueError(f"Grid2D does not support mode: {config.mode}")
        nx, ny = config.grid.nx, config.grid.ny
        dev = torch.device(device)
        self._empty = torch.empty(0, dtype=torch.float32, device=dev)
        # ping-pong halves; _cur selects the one holding the current state
        self._pairs = {f: [torch.zeros((nx, ny), dtype=torch.float32, device=dev) for _ in range(2)]
                       for f in _FIELDS[mode]}
        self._cur = 0
        shp = (nx, ny)
        self.eps_r, self.eps_inf, self.mu_r = np.ones(shp), np.ones(shp), np.ones(shp)
        self.sigma_e, self.sigma_m = np.zeros(shp), np.zeros(shp)
        self._version = 0
        # the maps start as ones and zeros: form those on the device directly
        one = torch.ones(shp, dtype=torch.float64, device=dev)
        self._form_coefficients(one, one, torch.zeros_like(one), torch.zeros_like(one))

    def _precompute_coefficients(self) -> None:
        """grid.py:157-195 in FP64, formed on the device: the material maps as
        they are now cross the host link once, and the four coefficient maps
        are computed there with the host formulas' operations in the same
        order (each one IEEE FP64 operation; the scalar divisions through
        physics.rdiv), so they equal the host formulas bit for bit.  Later
        edits of the maps take effect at the next call, as in the reference.
        ``_ca``, ``_cb``, ``_da`` and ``_db`` copy them to the host when read."""
        dev = self._empty.device
        f64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
        self._form_coefficients(f64(self.eps_inf), f64(self.mu_r), f64(self.sigma_e), f64(self.sigma_m))

    def _form_coefficients(self, eps_inf, mu_r, sigma_e, sigma_m) -> None:
        dt = self.config.dt
        eps = eps_inf * EPS_0
        mu = mu_r * MU_0
        se = sigma_e * dt / (2.0 * eps)
        sm = sigma_m * dt / (2.0 * mu)
        self._coef_dev = ((1.0 - se) / (1.0 + se), rdiv(dt, eps) / (1.0 + se),
                          (1.0 - sm) / (1.0 + sm), rdiv(dt, mu) / (1.0 + sm))
        self._coef_host = None
        self._version += 1

    def _host_coefficients(self):
        if self._coef_host is None:
            self._coef_host = tuple(t.cpu().numpy() for t in self._coef_dev)
        return self._coef_host

    _ca = property(lambda self: self._host_coefficients()[0])
    _cb = property(lambda self: self._host_coefficients()[1])
    _da = property(lambda self: self._host_coefficients()[2])
    _db = property(lambda self: self._host_coefficients()[3])

    def set_material_region(self, x_start, x_end, y_start, y_end, eps_r=1.0, mu_r=1.0, sigma_e=0.0, sigma_m=0.0,
                            eps_inf=None, debye_poles=None) -> None:
        if eps_r < 1.0:
            raise ValueError(f"Relative permittivity must be ≥ 1.0, got {eps_r}")
        if mu_r < 1.0:
            raise ValueError(f"Relative permeability must be ≥ 1.0, got {mu_r}")
        if sigma_e < 0.0:
            raise ValueError(f"Electric conductivity must be ≥ 0.0, got {sigma_e}")
        if debye_poles:
            raise NotImplementedError("dispersive materials are not supported by this solver")
        r = (slice(x_start, x_end), slice(y_start, y_end))
        self.eps_r[r], self.eps_inf[r] = eps_r, eps_r if eps_inf is None else eps_inf
        self.mu_r[r], self.sigma_e[r], self.sigma_m[r] = mu_r, sigma_e, sigma_m
        self._precompute_coefficients()

    def set_material_circle(self, center_x, center_y, radius, eps_r=1.0, mu_r=1.0, sigma_e=0.0, sigma_m=0.0,
                            eps_inf=None, debye_poles=None) -> None:
        if eps_r < 1.0:
            raise ValueError(f"Relative permittivity must be ≥ 1.0, got {eps_r}")
        if debye_poles:
            raise NotImplementedError("dispersive materials are not supported by this solver")
        nx, ny = self.config.grid.nx, self.config.grid.ny
        y_g, x_g = np.meshgrid(np.arange(ny), np.arange(nx))
        m = (x_g - center_x) ** 2 + (y_g - center_y) ** 2 <= radius ** 2
        self.eps_r[m], self.eps_inf[m] = eps_r, eps_r if eps_inf is None else eps_inf
        self.mu_r[m], self.sigma_e[m], self.sigma_m[m] = mu_r, sigma_e, sigma_m
        self._precompute_coefficients()

    def _field(self, name):
        pair = self._pairs.get(name)
        return self._empty if pair is None else pair[self._cur]

    ez = property(lambda self: self._field("ez"))
    hx = property(lambda self: self._field("hx"))
    hy = property(lambda self: self._field("hy"))
    hz = property(lambda self: self._field("hz"))
    ex = property(lambda self: self._field("ex"))
    ey = property(lambda self: self._field("ey"))

    def reset_fields(self) -> None:
        for pair in self._pairs.values():
            for t in pair:
                t.zero_()

    @property
    def memory_usage_bytes(self) -> int:
        return 11 * self.config.grid.total_cells * 8


class _Desc2S(C.Structure):
    P = C.c_void_p
    I = C.c_int32
    F = C.c_float
    _fields_ = [("nx", I), ("ny", I), ("mode", I), ("nsteps", I), ("inv_dx", F), ("inv_dy", F),
                ("dt_mu0", F), ("dt_eps0", F), ("mur_kx", F), ("mur_ky", F),
                ("f0", P * 2), ("f1", P * 2), ("f2", P * 2), ("coef_e", P), ("coef_h", P),
                ("n_ops", I), ("ops", I * 4), ("cpml_t", I), ("cpml", P), ("psi_e", P), ("psi_h", P * 2),
                ("mur_prev", P),
                ("nsrc", I), ("hz_sources", I), ("src", P), ("src_row", P), ("waveform", P),
                ("nrec", I), ("rec", P), ("rec_out", P), ("snap_field", I), ("snap_interval", I),
                ("snapshots", P)]


# -- solver (fdtd_2d.py, fdtd_base.py) -------------------------------------------------
class FDTD2D:
    """2D FDTD solver, TMz or TEz, on the device."""

    def __init__(self, config, sources: Optional[List] = None, boundaries: Optional[List] = None,
                 record_field: Optional[str] = None, record_interval: int = 1,
                 probe_points: Optional[List[Tuple[int, int]]] = None, dft_monitors: Optional[List] = None,
                 *, device: str = "cuda", use_graph: bool = True):
        self.config = config
        self.sources = list(sources or [])
        self.boundaries = list(boundaries or [])
        self.record_field = record_field
        self.record_interval = int(record_interval)
        self.probe_points = [tuple(int(v) for v in p) for p in (probe_points or [])]
        self.dft_monitors = list(dft_monitors or [])
        self.device = torch.device(device)
        self.use_graph = bool(use_graph)
        self._mode = _mode_name(config)
        self._validate()
        self.initialize(config)

    # -- set-up -------------------------------------------------------------------------
    def _validate(self):
        mode, g = self._mode, self.config.grid
        if mode not in _FIELDS:
            raise NotImplementedError(f"Solver not implemented for mode {self.config.mode}")
        nx, ny = g.nx, g.ny
        if nx < 3 or ny < 3:
            raise ValueError("grid must be at least 3x3")
        rec = self.record_field or "Ez"
        if self.probe_points and rec not in _COMP[mode]:
            raise ValueError(f"probes record {rec!r}, which a {mode} grid does not have")
        if self.record_field and self.record_field not in _COMP[mode]:
            raise ValueError(f"record_field {self.record_field!r} is not a {mode} component")
        for p in self.probe_points:
            if not (0 <= p[0] < nx and 0 <= p[1] < ny):
                raise ValueError(f"probe {p} outside the {nx}x{ny} grid")
        for s in self.sources:
            x, y = s.position
            if not (0 <= x < nx and 0 <= y < ny):
                raise ValueError(f"source at {(x, y)} outside the {nx}x{ny} grid")
            if s.component in ("Ex", "Ey") and mode == "TMZ":
                raise ValueError(f"a {s.component} source needs a TEz grid")
        for m in self.dft_monitors:
            if m.component not in _COMP[mode]:
                raise ValueError(f"monitor component {m.component!r} is not a {mode} component")
        kinds = [type(b).__name__ for b in self.boundaries]
        for k in kinds:
            if k not in ("CPML", "PEC", "MurABC"):
                raise NotImplementedError(f"boundary {k} is not supported")
        if kinds.count("CPML") > 1:
            raise NotImplementedError("one CPML per solver")
        if "MurABC" in kinds and kinds.index("MurABC") != len(kinds) - 1:
            raise NotImplementedError("MurABC must be the last boundary")
        if len(kinds) > 4:
            raise NotImplementedError("at most four boundaries")

    def initialize(self, config) -> None:
        self.config = config
        self.grid = Grid2D(config, self.device)
        self._step = 0
        self.field_snapshots: List[np.ndarray] = []
        self.probe_data: Dict[Tuple[int, int], List[float]] = {pt: [] for pt in self.probe_points}
        self._plan = None
        self._cap = 0
        self._coef_version = -1
        g, dev = config.grid, self.device
        nx, ny = g.nx, g.ny
        f32 = dict(dtype=torch.float32, device=dev)
        self._coef_e = torch.zeros((nx, ny, 2), **f32)
        self._coef_h = torch.zeros((nx, ny, 2), **f32)
        cp = next((b for b in self.boundaries if type(b).__name__ == "CPML"), None)
        self._cpml_t = int(cp.thickness) if cp is not None else 0
        t = max(self._cpml_t, 1)
        self._psi_e = torch.zeros(2 * t * ny + 2 * nx * t, **f32)
        self._psi_h = [torch.zeros(2 * t * ny + 2 * nx * t, **f32) for _ in range(2)]
        if cp is not None:
            kw = (cp.order, cp.sigma_factor, cp.alpha_max, cp.kappa_max)
            ax = cpml_coefficients(t, g.dx, config.dt, *kw)
            ay = cpml_coefficients(t, g.dy, config.dt, *kw)
            self._cpml = torch.as_tensor(np.concatenate(ax + ay), dtype=torch.float32).to(dev)
        else:
            self._cpml = torch.zeros(8, **f32)
        self._mur = torch.zeros(2 * (2 * ny + 2 * nx), **f32)
        # recorded cells: probes, then each monitor's region
        mode = self._mode
        cells = np.arange(nx * ny).reshape(nx, ny)
        rec = [(int(cells[p[0], p[1]]), _COMP[mode][self.record_field or "Ez"]) for p in self.probe_points]
        self._mon_slices = []
        for m in self.dft_monitors:
            idx = np.asarray(cells[m.region]).reshape(-1)
            self._mon_slices.append((len(rec), len(idx), np.shape(cells[m.region])))
            rec += [(int(c), _COMP[mode][m.component]) for c in idx]
        self._rec = torch.as_tensor(np.array(rec, np.int32).reshape(-1, 2)).to(dev)
        self._nrec = len(rec)
        # sources on the grid's components, stable-sorted by x
        keep = [s for s in self.sources if s.component in _COMP[mode] and s.component in ("Ez", "Hz", "Ex", "Ey")]
        order = sorted(range(len(keep)), key=lambda k: keep[k].position[0])
        self._src_objs = [keep[k] for k in order]
        src = np.array([[s.position[0], s.position[1], _COMP[mode][s.component]] for s in self._src_objs],
                       np.int32).reshape(-1, 3)
        row = np.zeros(nx + 1, np.int32)
        np.add.at(row, src[:, 0] + 1, 1)
        self._src = torch.as_tensor(src).to(dev)
        self._src_row = torch.as_tensor(np.cumsum(row).astype(np.int32)).to(dev)
        self._hz_src = int(mode == "TEZ" and bool((src[:, 2] == 0).any()))
        self._ops = [{"CPML": 1, "PEC": 2, "MurABC": 3}[type(b).__name__] for b in self.boundaries]

    def _fields(self):
        return [self.grid._pairs[f] for f in _FIELDS[self._mode]]

    def _ensure(self, end: int) -> None:
        """Plan covering steps [0, end): waveform table, record and snapshot
        buffers sized to the capacity (grown by doubling; recorded values and
        all field / boundary state are kept)."""
        if self._plan is not None and end <= self._cap:
            return
        cap = max(end, self.config.num_steps, 2 * self._cap)
        dt = self.config.dt
        dev = self.device
        w = np.array([[s.value_at(n, dt) for n in range(cap)] for s in self._src_objs], np.float64)
        self._wave = torch.as_tensor(w.reshape(len(self._src_objs), cap), dtype=torch.float32).to(dev)
        rec_out = torch.zeros((max(self._nrec, 1), cap), dtype=torch.float32, device=dev)
        if self._plan is not None:
            rec_out[:, :self._cap] = self._rec_out[:, :self._cap]
        self._rec_out = rec_out
        g = self.config.grid
        old = getattr(self, "_snaps", None)
        self._snaps = None
        if self.record_field:
            nsnap = (cap + self.record_interval - 1) // self.record_interval
            self._snaps = torch.zeros((nsnap, g.nx, g.ny), dtype=torch.float32, device=dev)
            if old is not None and self._plan is not None:
                self._snaps[:len(old)] = old
        if self._plan is not None:
            lib().ceep2s_plan_destroy(self._plan)
        d = _Desc2S()
        d.nx, d.ny, d.mode, d.nsteps = g.nx, g.ny, 0 if self._mode == "TMZ" else 1, cap
        d.inv_dx, d.inv_dy = 1.0 / g.dx, 1.0 / g.dy
        d.dt_mu0, d.dt_eps0 = dt / MU_0, dt / EPS_0
        cdt = C_0 * dt
        d.mur_kx, d.mur_ky = (cdt - g.dx) / (cdt + g.dx), (cdt - g.dy) / (cdt + g.dy)
        f = self._fields()
        for k in range(2):
            d.f0[k], d.f1[k], d.f2[k] = f[0][k].data_ptr(), f[1][k].data_ptr(), f[2][k].data_ptr()
            d.psi_h[k] = self._psi_h[k].data_ptr()
        d.coef_e, d.coef_h = self._coef_e.data_ptr(), self._coef_h.data_ptr()
        d.n_ops = len(self._ops)
        for k, op in enumerate(self._ops):
            d.ops[k] = op
        d.cpml_t, d.cpml, d.psi_e, d.mur_prev = self._cpml_t, self._cpml.data_ptr(), self._psi_e.data_ptr(), \
            self._mur.data_ptr()
        d.nsrc, d.hz_sources = len(self._src_objs), self._hz_src
        if self._src_objs:
            d.src, d.src_row, d.waveform = self._src.data_ptr(), self._src_row.data_ptr(), self._wave.data_ptr()
        d.nrec = self._nrec
        if self._nrec:
            d.rec, d.rec_out = self._rec.data_ptr(), self._rec_out.data_ptr()
        if self._snaps is not None:
            d.snap_field, d.snap_interval = _COMP[self._mode][self.record_field], self.record_interval
            d.snapshots = self._snaps.data_ptr()
        plan = C.c_void_p()
        check(lib().ceep2s_plan_create(C.addressof(d), C.byref(plan)), "ceep2s_plan_create")
        check(lib().ceep2s_plan_set_current_buffer(plan, self.grid._cur), "ceep2s_plan_set_current_buffer")
        self._plan, self._cap = plan, cap

    def _upload_coefficients(self) -> None:
        g = self.grid
        if self._coef_version == g._version:
            return
        ca, cb, da, db = g._coef_dev
        self._coef_e.copy_(torch.stack([ca, cb], -1))      # FP64 -> FP32, rounded to nearest
        self._coef_h.copy_(torch.stack([da, db], -1))
        self._coef_version = g._version

    def __del__(self):
        if getattr(self, "_plan", None) is not None:
            try:
                lib().ceep2s_plan_destroy(self._plan)
            except Exception:
                pass
            self._plan = None

    # -- time stepping (fdtd_base.py:158-210) ---------------------------------------------
    def advance(self, num_steps: int, stream=None) -> None:
        """Run ``num_steps`` steps on the device without the host-side
        bookkeeping (probe lists, snapshots, monitors): call ``collect()``."""
        if num_steps <= 0:
            return
        self._upload_coefficients()
        a = self._step
        self._ensure(a + num_steps)
        s = torch.cuda.current_stream(self.device) if stream is None else stream
        check(lib().ceep2s_plan_run(self._plan, a, num_steps, C.c_void_p(s.cuda_stream), int(self.use_graph)),
              "ceep2s_plan_run")
        self.grid._cur = lib().ceep2s_plan_current_buffer(self._plan)
        self._step += num_steps
        self._pending = getattr(self, "_pending", 0) + num_steps

    def collect(self) -> None:
        """Move the recorded steps not yet collected to the host containers."""
        n = getattr(self, "_pending", 0)
        if n == 0:
            return
        a, b = self._step - n, self._step
        if self._nrec:
            vals = self._rec_out[:, a:b].double()
            host = vals[:len(self.probe_points)].cpu().numpy()
            for k, pt in enumerate(self.probe_points):
                self.probe_data[pt].extend(host[k].tolist())
            dt = self.config.dt
            for m, (off, cnt, shp) in zip(self.dft_monitors, self._mon_slices):
                ser = vals[off:off + cnt]                                   # (cells, n)
                tt = torch.arange(a, b, dtype=torch.float64, device=self.device) * dt
                om = torch.as_tensor(m.omega if hasattr(m, "omega") else 2 * np.pi * np.asarray(m.frequencies),
                                     dtype=torch.float64, device=self.device)
                ph = om[:, None] * tt[None, :]
                re = (torch.cos(ph) @ ser.t() * dt).cpu().numpy()
                im = (-torch.sin(ph) @ ser.t() * dt).cpu().numpy()
                nf = len(om)
                if getattr(m, "dft_real", None) is None:
                    m.dft_real = np.zeros((nf,) + tuple(shp))
                    m.dft_imag = np.zeros((nf,) + tuple(shp))
                    m._initialized = True
                m.dft_real += re.reshape((nf,) + tuple(shp))
                m.dft_imag += im.reshape((nf,) + tuple(shp))
        if self._snaps is not None:
            first = (a + self.record_interval - 1) // self.record_interval
            last = (b - 1) // self.record_interval
            for k in range(first, last + 1):
                self.field_snapshots.append(self._snaps[k].cpu().numpy().astype(np.float64))
        self._pending = 0

    def reset(self) -> None:
        """Zero every field, psi and Mur state and start again at step 0 with
        empty probe lists and snapshots (not in the reference; reuses buffers
        and captured graphs)."""
        self.grid.reset_fields()
        self._psi_e.zero_()
        for t in self._psi_h:
            t.zero_()
        self._mur.zero_()
        self._step, self._pending = 0, 0
        self.field_snapshots = []
        self.probe_data = {pt: [] for pt in self.probe_points}
        for m in self.dft_monitors:
            m.dft_real = m.dft_imag = None
            m._initialized = False

    def step(self) -> None:
        """One step (H, H boundaries, E, sources, E boundaries, record)."""
        self.advance(1)
        self.collect()

    def run(self, num_steps: Optional[int] = None) -> None:
        if num_steps is None:
            num_steps = self.config.num_steps
        self.advance(num_steps)
        self.collect()

    # -- accessors ---------------------------------------------------------------------------
    @property
    def current_step(self) -> int:
        return self._step

    @property
    def current_time(self) -> float:
        return self._step * self.config.dt

    def get_field(self, component: str) -> torch.Tensor:
        fmap = {"Ez": self.grid.ez, "Hx": self.grid.hx, "Hy": self.grid.hy,
                "Hz": self.grid.hz, "Ex": self.grid.ex, "Ey": self.grid.ey}
        if component not in fmap:
            raise ValueError(f"Unknown component '{component}'. Use: {list(fmap)}")
        return fmap[component]
