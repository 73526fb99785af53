"""Drop-in ``BatchedFDTD3D`` backed by the sm_100a kernels.

Keeps the constructor, attributes and methods of the reference class
(src/ceep/solvers/fdtd_3d_batched.py:48-1011): ``set_material_region``,
``set_material_sphere``, ``set_phantom``, ``run(verbose)`` returning
``{tx: {rx: float64 series}}``, ``compute_energy()``.  Keyword-only
extensions: ``waveform``, ``frequencies`` + ``s_matrix()``, ``set_dispersion``,
``device``.  Divergences: positions are validated up front (ValueError), the
arithmetic is FP32 on the device, state tensors are torch CUDA tensors.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import physics, trace
from ._lib import Desc3D, check, lib
from .constants import EPS_0, MU_0, cfl_timestep_3d
from .solvers import PinnedMaps, _pad_tx, _ptr


class BatchedFDTD3D:
    """Batched 3D Yee FDTD, one transmit event per batch element (z-directed sources)."""

    def __init__(self, nx: int, ny: int, nz: int, dx: float, total_steps: int, cpml_thickness: int,
                 source_positions: List[Tuple[int, int, int]], probe_positions: List[Tuple[int, int, int]],
                 frequency: float, delay_factor: float = 5.0, *, waveform: Optional[np.ndarray] = None,
                 frequencies: Optional[Sequence[float]] = None, device: str = "cuda", z_rows: int = 0,
                 shell_z_rows: int = 0,
                 use_graph: bool = True):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dx = self.dy = self.dz = float(dx)
        self.total_steps = int(total_steps)
        self.cpml_thickness = int(cpml_thickness)
        self.source_positions = [tuple(int(v) for v in p) for p in source_positions]
        self.probe_positions = [tuple(int(v) for v in p) for p in probe_positions]
        self.frequency = float(frequency)
        self.delay_factor = float(delay_factor)
        self.batch = len(self.source_positions)
        self.dt = cfl_timestep_3d(dx, dx, dx, courant=0.5) * 0.99          # fdtd_3d_batched.py:133
        shp = (nx, ny, nz)
        self._eps_r = np.ones(shp)
        self._sigma_e = np.zeros(shp)
        self._mu_r = np.ones(shp)
        self._sigma_m = np.zeros(shp)
        self._debye: list = []
        self._lorentz: list = []
        self._waveform_override = None if waveform is None else np.asarray(waveform, np.float64)
        self.frequencies = None if frequencies is None else np.asarray(frequencies, np.float64)
        self.device = torch.device(device)
        self.z_rows = int(z_rows)
        self.shell_z_rows = int(shell_z_rows)
        self.use_graph = bool(use_graph)
        self._pins: Optional[PinnedMaps] = None      # page-locked map storage once built on a GPU
        self.run_record: Optional[dict] = None       # last run's record (ceep_b200.trace)
        self.record_path: Optional[str] = None       # append each run's record as a JSON line
        self._built = False
        self._plan = None
        n = self.cpml_thickness
        if self.batch < 1:
            raise ValueError("at least one source position is required")
        if n < 0 or n == 1:
            raise ValueError("cpml_thickness must be 0 or >= 2")
        if min(nx, ny, nz) < 2 * n + 2:
            raise ValueError(f"grid {nx}x{ny}x{nz} must exceed twice the CPML thickness ({n}) by 2")
        for kind, pts in (("source", self.source_positions), ("probe", self.probe_positions)):
            for p in pts:
                if len(p) != 3 or not all(0 <= v < m for v, m in zip(p, shp)):
                    raise ValueError(f"{kind} position {p} outside the {nx}x{ny}x{nz} grid")

    # -- materials (fdtd_3d_batched.py:143-264) ------------------------------
    def set_material_region(self, x_start, x_end, y_start, y_end, z_start, z_end, eps_r=1.0, sigma_e=0.0,
                            mu_r=1.0, sigma_m=0.0) -> None:
        r = (slice(x_start, x_end), slice(y_start, y_end), slice(z_start, z_end))
        self._eps_r[r], self._sigma_e[r], self._mu_r[r], self._sigma_m[r] = eps_r, sigma_e, mu_r, sigma_m

    def set_material_sphere(self, center_x, center_y, center_z, radius, eps_r=1.0, sigma_e=0.0, mu_r=1.0,
                            sigma_m=0.0) -> None:
        """As fdtd_3d_batched.py:213-225: the mask is built on a meshgrid over
        (nz, ny, nx), so the call only works on cubic grids (IndexError
        otherwise, like the reference) and the sphere's x and z centres swap."""
        zg, yg, xg = np.meshgrid(np.arange(self.nz), np.arange(self.ny), np.arange(self.nx), indexing="ij")
        mask = (xg - center_x) ** 2 + (yg - center_y) ** 2 + (zg - center_z) ** 2 <= radius ** 2
        self._eps_r[mask], self._sigma_e[mask], self._mu_r[mask], self._sigma_m[mask] = eps_r, sigma_e, mu_r, sigma_m

    def set_phantom(self, phantom) -> None:
        """fdtd_3d_batched.py:227-264 duck typing; ``get_dispersion()`` adds ADE poles."""
        if hasattr(phantom, "get_eps_map_3d"):
            e, s = phantom.get_eps_map_3d(self.frequency)
            self._eps_r[:], self._sigma_e[:] = e, s
        elif hasattr(phantom, "get_eps_map"):
            e, s = phantom.get_eps_map(self.frequency)
            self._eps_r[:] = np.asarray(e)[:, :, None]
            self._sigma_e[:] = np.asarray(s)[:, :, None]
        elif hasattr(phantom, "get_permittivity_map"):
            er, ei = phantom.get_permittivity_map(self.frequency)
            self._eps_r[:] = np.asarray(er)[:, :, None]
            self._sigma_e[:] = (np.asarray(ei) * 2 * np.pi * self.frequency * EPS_0)[:, :, None]
        elif hasattr(phantom, "eps_r"):
            self._eps_r[:] = phantom.eps_r
            if hasattr(phantom, "sigma_e"):
                self._sigma_e[:] = phantom.sigma_e
        else:
            raise TypeError("Phantom must have get_eps_map_3d(), get_eps_map(), get_permittivity_map(), "
                            "or eps_r attribute")
        if hasattr(phantom, "get_dispersion"):
            d = phantom.get_dispersion()
            self.set_dispersion(debye=d.get("debye", ()), lorentz=d.get("lorentz", ()))

    def set_dispersion(self, debye=(), lorentz=()) -> None:
        """Debye ``(delta_eps, tau)`` / Lorentz ``(delta_eps, omega_0, delta)`` maps
        (nx, ny, nz) acting on every E component inside the E interior box."""
        if self._built and (len(debye), len(lorentz)) != (len(self._debye), len(self._lorentz)):
            raise RuntimeError("the number of poles cannot change after the first run()")
        if len(debye) + len(lorentz) > 2:
            raise ValueError("at most two ADE poles per cell are compiled in")
        shp = (self.nx, self.ny, self.nz)
        n = self.cpml_thickness
        inner = np.zeros(shp, bool)
        inner[n + 1:self.nx - n, n + 1:self.ny - n, n + 1:self.nz - n] = True
        keep = ((lambda key, a: self._pins.hold(key, a, shp)) if self._pins is not None
                else (lambda key, a: np.broadcast_to(np.asarray(a, np.float64), shp).copy()))
        deb = [tuple(keep(("debye", i, j), a) for j, a in enumerate(p)) for i, p in enumerate(debye)]
        lor = [tuple(keep(("lorentz", i, j), a) for j, a in enumerate(p)) for i, p in enumerate(lorentz)]
        for p in deb + lor:
            if np.any((p[1] > 0) & (p[0] != 0) & ~inner):
                raise ValueError("ADE pole present outside the interior E region")
        self._debye, self._lorentz = deb, lor

    # -- build ---------------------------------------------------------------
    def _coef_maps(self):
        """Device (nz, ny, nx, 4) float32 (da, db, ca, cb) and (poles, nz, ny,
        nx, 4) ADE coefficients (fdtd_3d_batched.py:281-296), computed in FP64
        on the device with the host formulas (bit-identical)."""
        return physics.coefficient_tensors_3d(self._eps_r, self._sigma_e, self._mu_r, self._sigma_m, self.dt,
                                              self._debye, self._lorentz, self.device)

    def _build(self):
        dev = self.device
        if dev.type != "cuda" or not torch.cuda.is_available():
            raise RuntimeError("BatchedFDTD3D needs a CUDA device (B200); there is no CPU path")
        lib()
        nx, ny, nz, n, B = self.nx, self.ny, self.nz, self.cpml_thickness, self.batch
        BP = _pad_tx(B)
        G = BP // min(BP, 32)
        W = BP // G
        self.ntx_pad, self._groups, self._gwidth = BP, G, W
        f32 = dict(dtype=torch.float32, device=dev)
        to_dev = lambda a, dt_=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt_).to(dev)
        # from here on the maps live in page-locked memory (update_materials copies them)
        self._pins = PinnedMaps()
        for name in ("_eps_r", "_sigma_e", "_mu_r", "_sigma_m"):
            setattr(self, name, self._pins.hold(name, getattr(self, name)))
        self._debye = [tuple(self._pins.hold(("debye", i, j), a) for j, a in enumerate(p))
                       for i, p in enumerate(self._debye)]
        self._lorentz = [tuple(self._pins.hold(("lorentz", i, j), a) for j, a in enumerate(p))
                         for i, p in enumerate(self._lorentz)]
        coef, ade = self._coef_maps()
        self._coef = coef
        self._ade_coef = ade if ade.shape[0] else None
        b, c = physics.cpml_profile(n, self.dx, self.dt)
        self._cpml_b, self._cpml_c = to_dev(b if n else np.zeros(1)), to_dev(c if n else np.zeros(1))
        w = (self._waveform_override if self._waveform_override is not None
             else physics.gaussian_derivative(self.total_steps, self.dt, self.frequency, self.delay_factor))
        self.waveform = to_dev(w)
        F = lambda: torch.zeros((G, nz, ny, nx, W), **f32)
        self._f = {k: F() for k in ("ex", "ey", "ez", "hx", "hy", "hz")}
        nn = max(n, 1)
        self._psi = {k: torch.zeros((G, nz, ny, 2 * nn, W), **f32) for k in ("hxy", "hzy")}
        self._psi.update({k: torch.zeros((G, nz, 2 * nn, nx, W), **f32) for k in ("hyx", "hzx")})
        self._psi.update({k: torch.zeros((G, 2 * nn, ny, nx, W), **f32) for k in ("hxz", "hyz")})
        nd, nl = len(self._debye), len(self._lorentz)
        self._j = torch.zeros((G, nd + nl, 3, nz, ny, nx, W), **f32) if nd + nl else None
        self._j_prev = torch.zeros((G, nl, 3, nz, ny, nx, W), **f32) if nl else None
        P = len(self.probe_positions)
        self._src = to_dev(np.array(self.source_positions, np.int32).reshape(-1, 3), torch.int32)
        self._prb = to_dev(np.array(self.probe_positions, np.int32).reshape(-1, 3), torch.int32)
        self.probe_data = torch.zeros((B, max(P, 1), self.total_steps), **f32)
        d = Desc3D()
        d.nx, d.ny, d.nz, d.cpml, d.ntx, d.ntx_pad = nx, ny, nz, n, B, BP
        d.nprobe, d.nsteps, d.n_debye, d.n_lorentz = P, self.total_steps, nd, nl
        d.inv_dx, d.dt = 1.0 / self.dx, self.dt
        for k, t in self._f.items():
            setattr(d, k, _ptr(t))
        for k, t in self._psi.items():
            setattr(d, "psi_" + k, _ptr(t))
        d.j, d.j_prev = _ptr(self._j), _ptr(self._j_prev)
        d.coef, d.ade_coef = _ptr(self._coef), _ptr(self._ade_coef)
        d.cpml_b, d.cpml_c = _ptr(self._cpml_b), _ptr(self._cpml_c)
        d.src_xyz, d.prb_xyz = _ptr(self._src), _ptr(self._prb)
        d.waveform, d.probes = _ptr(self.waveform), _ptr(self.probe_data)
        d.z_rows = self.z_rows
        d.shell_z_rows = self.shell_z_rows
        self._desc = d
        plan = C.c_void_p()
        check(lib().ceep3d_plan_create(C.byref(d), C.byref(plan)), "ceep3d_plan_create")
        self._plan = plan
        self._built = True

    def __del__(self):
        if getattr(self, "_plan", None) is not None:
            try:
                lib().ceep3d_plan_destroy(self._plan)
            except Exception:
                pass
            self._plan = None

    # -- time loop -----------------------------------------------------------
    def advance(self, step0: int = 0, nsteps: Optional[int] = None, stream=None) -> None:
        if not self._built:
            self._build()
        nsteps = self.total_steps - step0 if nsteps is None else nsteps
        s = torch.cuda.current_stream(self.device) if stream is None else stream
        check(lib().ceep3d_plan_run(self._plan, step0, nsteps, C.c_void_p(s.cuda_stream), int(self.use_graph)),
              "ceep3d_plan_run")

    def run(self, verbose: bool = False) -> Dict[int, Dict[int, np.ndarray]]:
        """fdtd_3d_batched.py:886-985; with ``verbose`` prints the throughput line."""
        t0 = time.perf_counter()
        with trace.phase("time_loop"):
            self.advance(0, self.total_steps)
            probe_np = self.probe_data.double().cpu().numpy()
        trace.emit(self, trace.make_record("BatchedFDTD3D", self.nx * self.ny * self.nz, self.total_steps,
                                           self.batch, time.perf_counter() - t0))
        if verbose:
            el = time.perf_counter() - t0
            rate = self.batch * self.nx * self.ny * self.nz * self.total_steps / el / 1e9
            print(f"\nCompleted {self.total_steps} steps in {el:.2f}s")
            print(f"Performance: {rate:.2f} G cell-updates/sec")
        P = len(self.probe_positions)
        return {tx: {rx: probe_np[tx, rx, :] for rx in range(P)} for tx in range(self.batch)}

    def s_matrix(self, frequencies: Optional[Sequence[float]] = None) -> np.ndarray:
        freqs = self.frequencies if frequencies is None else np.asarray(frequencies, np.float64)
        if freqs is None:
            raise ValueError("no frequencies given")
        from .spectral import dft
        with trace.phase("dft"):
            return dft(self.probe_data[:, :len(self.probe_positions)], freqs,
                       self.dt).cpu().numpy().astype(np.complex128)

    def _ref_view(self, t):
        G, nz, ny, nx, W = t.shape
        v = t.permute(0, 4, 3, 2, 1)                    # (G, W, nx, ny, nz)
        v = v.reshape(G * W, nx, ny, nz) if G > 1 else v[0]
        return v[:self.batch]

    def __getattr__(self, name):
        if name in ("ex", "ey", "ez", "hx", "hy", "hz"):
            f = self.__dict__.get("_f")
            return None if f is None else self._ref_view(f[name])
        raise AttributeError(name)

    def reset(self) -> None:
        """Zero all field, psi and ADE state (not in the reference; reuses buffers)."""
        if not self._built:
            return
        for t in list(self._f.values()) + list(self._psi.values()) + [self._j, self._j_prev, self.probe_data]:
            if t is not None:
                t.zero_()

    def material_tensors(self, eps_r, sigma_e, debye=(), lorentz=()):
        """Device (coef, ade) tensors for the given maps, for ``load_material_tensors``."""
        saved = (self._eps_r, self._sigma_e, self._debye, self._lorentz)
        try:
            self._eps_r, self._sigma_e = np.asarray(eps_r, np.float64), np.asarray(sigma_e, np.float64)
            self._debye, self._lorentz = list(debye), list(lorentz)
            coef, ade = self._coef_maps()
        finally:
            self._eps_r, self._sigma_e, self._debye, self._lorentz = saved
        return coef, (ade if ade.shape[0] else None)

    def load_material_tensors(self, mats) -> None:
        if not self._built:
            self._build()
        coef, ade = mats
        if (ade is None) != (self._ade_coef is None):
            raise ValueError("ADE pole count differs from the built solver")
        self._coef.copy_(coef, non_blocking=True)
        if ade is not None:
            self._ade_coef.copy_(ade, non_blocking=True)

    def update_materials(self) -> None:
        if not self._built:
            return
        coef, ade = self._coef_maps()
        self._coef.copy_(coef)
        if ade.shape[0]:
            self._ade_coef.copy_(ade)

    def compute_energy(self) -> float:
        """fdtd_3d_batched.py:987-1011 (sums in FP64 on the device)."""
        if not self._built:
            return 0.0
        sq = lambda k: float(self._ref_view(self._f[k]).double().pow(2).sum())
        e = 0.5 * EPS_0 * (sq("ex") + sq("ey") + sq("ez"))
        h = 0.5 * MU_0 * (sq("hx") + sq("hy") + sq("hz"))
        return (e + h) * self.dx * self.dy * self.dz
