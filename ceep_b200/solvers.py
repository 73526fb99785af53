"""Drop-in batched solvers backed by the sm_100a kernels.

``BatchedFDTD2D`` keeps the constructor, attributes and methods of the
reference class (src/ceep/solvers/fdtd_2d_batched.py:41-611) so callers such
as dataset generators switch by changing the import.  Differences, all
documented on the methods:

* positions are validated up front (ValueError) instead of wrapping or
  failing inside the loop;
* arithmetic is FP32 on the device (the reference is FP64);
* ``probe_data``, ``ez``, ``hx``, ``hy`` are torch CUDA tensors (the
  reference exposes CuPy arrays); ``run()`` still returns host float64 series;
* keyword-only extensions (defaults reproduce the reference): ``courant``,
  ``cpml_R0``, ``cpml_order``, ``waveform``, ``frequencies`` (S-matrix),
  ``set_dispersion`` (Debye/Lorentz ADE), ``device``.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import physics, trace
from ._lib import Desc2D, check, lib
from .constants import C_0, EPS_0, MU_0


def _pad_tx(ntx: int) -> int:
    if ntx <= 4:
        return 4
    if ntx <= 8:
        return 8
    if ntx <= 16:
        return 16
    return 32 * ((ntx + 31) // 32)


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


class PinnedMaps:
    """Page-locked host storage for the FP64 material maps of a solver that
    runs on a CUDA device.  The maps are the one host-to-device transfer of a
    material update (``update_materials``); from page-locked memory that copy
    runs at the link's full rate instead of through the driver's staging
    buffers.  ``hold`` returns a NumPy view of a page-locked buffer (kept per
    key and reused while the shape stays) holding a copy of `arr`."""

    def __init__(self):
        self._bufs = {}

    def hold(self, key, arr, shape=None) -> np.ndarray:
        a = np.asarray(arr, np.float64)
        shape = a.shape if shape is None else tuple(shape)
        t = self._bufs.get(key)
        if t is None or tuple(t.shape) != shape:
            t = torch.empty(shape, dtype=torch.float64, pin_memory=True)
            self._bufs[key] = t
        out = t.numpy()
        if a.shape == shape and a.flags.c_contiguous:
            t.copy_(torch.from_numpy(a))    # a full map: torch's copy runs on several host threads
        else:
            np.copyto(out, np.broadcast_to(a, shape))
        return out


def fill_map(dst: np.ndarray, src) -> None:
    """``dst[:] = src``; a full C-contiguous FP64 map of dst's shape goes
    through torch's multithreaded host copy (a 600x600 map: 0.33 -> 0.10 ms)."""
    a = np.asarray(src)
    if (a.dtype == np.float64 and a.shape == dst.shape and a.flags.c_contiguous and dst.flags.c_contiguous
            and dst.flags.writeable):
        torch.from_numpy(dst).copy_(torch.from_numpy(a))
    else:
        dst[:] = a


class FDTDStatusError(RuntimeError):
    """A device status word reported a failure: CEEP_ERR_TIMEOUT (4, a bounded
    wait ran out) or CEEP_ERR_NONFINITE (5, the sentinel found NaN/Inf)."""
    TIMEOUT, NONFINITE = 4, 5

    def __init__(self, code: int):
        what = {4: "a bounded device wait expired", 5: "a NaN/Inf value was found by the sentinel"}
        super().__init__(f"fused step reported status {code} ({what.get(code, 'unknown')})")
        self.code = code


class BatchedFDTD2D:
    """Batched 2D TMz FDTD, one transmit event per batch element, shared materials.

    Parameters mirror fdtd_2d_batched.py:66-77.
    """

    def __init__(self, nx: int, ny: int, dx: float, total_steps: int, cpml_thickness: int,
                 source_positions: List[Tuple[int, int]], probe_positions: List[Tuple[int, int]],
                 frequency: float, delay_factor: float = 5.0, *, courant: Optional[float] = None,
                 cpml_R0: float = 1e-8, cpml_order: int = 3, waveform: Optional[np.ndarray] = None,
                 frequencies: Optional[Sequence[float]] = None, device: str = "cuda",
                 rows_per_block: int = 0, use_graph: bool = True, temporal_block: int = 2):
        self.nx, self.ny = int(nx), int(ny)
        self.dx = self.dy = float(dx)
        self.total_steps = int(total_steps)
        self.cpml_n = int(cpml_thickness)
        self.source_positions = [tuple(int(v) for v in p) for p in source_positions]
        self.probe_positions = [tuple(int(v) for v in p) for p in probe_positions]
        self.frequency = float(frequency)
        self.delay_factor = float(delay_factor)
        self.batch = len(self.source_positions)
        # CFL step of fdtd_2d_batched.py:92 unless a Courant number is given
        self.dt = dx / (C_0 * np.sqrt(2.0)) * 0.99 if courant is None else float(courant) * dx / C_0
        self._eps_r = np.ones((nx, ny), dtype=np.float64)
        self._sigma_e = np.zeros((nx, ny), dtype=np.float64)
        self._debye: list = []
        self._lorentz: list = []
        self.cpml_R0, self.cpml_order = float(cpml_R0), int(cpml_order)
        self._waveform_override = None if waveform is None else np.asarray(waveform, np.float64)
        self.frequencies = None if frequencies is None else np.asarray(frequencies, np.float64)
        self.device = torch.device(device)
        self.rows_per_block = int(rows_per_block)
        self.use_graph = bool(use_graph)
        self.temporal_block = int(temporal_block)   # steps per kernel launch (1 or 2)
        self.frame_split = False                     # two-step frame and interior tiles as two kernels
        self.sentinel_interval = 0                   # NaN/Inf scans between run-range ends (0: none)
        self.wait_limit_ns = 1_000_000_000           # bound of every device wait
        self._pins: Optional[PinnedMaps] = None      # page-locked map storage once built on a GPU
        self.run_record: Optional[dict] = None       # last run's record (ceep_b200.trace)
        self.record_path: Optional[str] = None       # append each run's record as a JSON line
        self._built = False
        self._plan = None
        self._validate()

    # -- validation (the reference silently wraps negative indices) ----------
    def _validate(self):
        n, nx, ny = self.cpml_n, self.nx, self.ny
        if self.batch < 1:
            raise ValueError("at least one source position is required")
        if n < 0 or n == 1:
            raise ValueError("cpml_thickness must be 0 or >= 2 (n = 1 divides by zero in the grading)")
        if nx < 2 * n + 2 or ny < 2 * n + 2:
            raise ValueError(f"grid {nx}x{ny} must exceed twice the CPML thickness ({n}) by 2")
        if self.total_steps < 1:
            raise ValueError("total_steps must be >= 1")
        for kind, pts in (("source", self.source_positions), ("probe", self.probe_positions)):
            for p in pts:
                if len(p) != 2 or not (0 <= p[0] < nx and 0 <= p[1] < ny):
                    raise ValueError(f"{kind} position {p} outside the {nx}x{ny} grid")
        if self._waveform_override is not None and self._waveform_override.shape != (self.total_steps,):
            raise ValueError("waveform must have total_steps samples")

    # -- materials (fdtd_2d_batched.py:100-136) ------------------------------
    def set_material_circle(self, center_x: int, center_y: int, radius: int, eps_r: float,
                            sigma_e: float = 0.0) -> None:
        x, y = np.meshgrid(np.arange(self.nx), np.arange(self.ny), indexing="ij")
        mask = (x - center_x) ** 2 + (y - center_y) ** 2 <= radius ** 2
        self._eps_r[mask] = eps_r
        self._sigma_e[mask] = sigma_e

    def set_phantom(self, phantom) -> None:
        """Same duck typing as fdtd_2d_batched.py:112-136 (TypeError otherwise).
        A phantom that also exposes ``get_dispersion()`` (Debye/Lorentz maps)
        sets the ADE poles as well."""
        if hasattr(phantom, "get_eps_map"):
            eps_r, sigma_e = phantom.get_eps_map(self.frequency)
            fill_map(self._eps_r, eps_r)
            fill_map(self._sigma_e, sigma_e)
        elif hasattr(phantom, "get_permittivity_map"):
            eps_real, eps_imag = phantom.get_permittivity_map(self.frequency)
            self._eps_r[:] = eps_real
            self._sigma_e[:] = eps_imag * (2 * np.pi * self.frequency) * EPS_0
        elif hasattr(phantom, "eps_r"):
            self._eps_r[:] = phantom.eps_r
            if hasattr(phantom, "sigma_e"):
                self._sigma_e[:] = phantom.sigma_e
        else:
            raise TypeError("Phantom must have get_eps_map(), get_permittivity_map(), or eps_r attribute")
        if hasattr(phantom, "get_dispersion"):
            d = phantom.get_dispersion()
            self.set_dispersion(debye=d.get("debye", ()), lorentz=d.get("lorentz", ()))

    def set_dispersion(self, debye=(), lorentz=()) -> None:
        """Debye poles ``(delta_eps, tau)`` and Lorentz poles ``(delta_eps, omega_0, delta)``
        as per-cell (nx, ny) maps or scalars; ``_eps_r`` then holds eps_inf.
        The ADE acts on the interior E region only, so every pole map must be zero
        in the CPML strips (ValueError otherwise)."""
        if self._built and (len(debye), len(lorentz)) != (len(self._debye), len(self._lorentz)):
            raise RuntimeError("the number of Debye/Lorentz poles cannot change after the first run(); "
                               "create a new solver")
        if len(debye) + len(lorentz) > 2:
            raise ValueError("at most two ADE poles per cell are compiled in")
        shp = (self.nx, self.ny)
        keep = ((lambda key, a: self._pins.hold(key, a, shp)) if self._pins is not None
                else (lambda key, a: np.broadcast_to(np.asarray(a, np.float64), shp).copy()))
        deb = [tuple(keep(("debye", i, j), a) for j, a in enumerate(p)) for i, p in enumerate(debye)]
        lor = [tuple(keep(("lorentz", i, j), a) for j, a in enumerate(p)) for i, p in enumerate(lorentz)]
        # the cells outside the interior E region [n+1, nx-n) x [n+1, ny-n):
        # two full-width row bands and two column bands between them
        n = self.cpml_n
        a0, a1, b0, b1 = n + 1, max(self.nx - n, n + 1), n + 1, max(self.ny - n, n + 1)
        outside = [(slice(0, a0), slice(None)), (slice(a1, None), slice(None)),
                   (slice(a0, a1), slice(0, b0)), (slice(a0, a1), slice(b1, None))]

        def present_outside(pole):
            return any(np.any((pole[1][r] > 0) & (pole[0][r] != 0)) for r in outside)
        for p in deb:
            if present_outside(p):
                raise ValueError("Debye pole present outside the interior E region")
        for p in lor:
            if present_outside(p):
                raise ValueError("Lorentz pole present outside the interior E region")
        self._debye, self._lorentz = deb, lor

    # -- build: host FP64 coefficients -> device FP32 (fdtd_2d_batched.py:138-270)
    def _build(self):
        dev = self.device
        if dev.type != "cuda" or not torch.cuda.is_available():
            raise RuntimeError("BatchedFDTD2D needs a CUDA device (B200); there is no CPU path")
        lib()
        nx, ny, n, B = self.nx, self.ny, self.cpml_n, self.batch
        BP = _pad_tx(B)
        self.ntx_pad = BP
        G = BP // min(BP, 32)           # TX groups of at most 32 (kernel grid.z)
        W = BP // G                     # floats per cell in one group
        self._groups, self._gwidth = G, W
        dt = self.dt
        f32 = dict(dtype=torch.float32, device=dev)
        # from here on the maps live in page-locked memory (update_materials copies them)
        self._pins = PinnedMaps()
        self._eps_r = self._pins.hold("eps_r", self._eps_r)
        self._sigma_e = self._pins.hold("sigma_e", self._sigma_e)
        self._debye = [tuple(self._pins.hold(("debye", i, j), a) for j, a in enumerate(p))
                       for i, p in enumerate(self._debye)]
        self._lorentz = [tuple(self._pins.hold(("lorentz", i, j), a) for j, a in enumerate(p))
                         for i, p in enumerate(self._lorentz)]
        to_dev = lambda a, dt_=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt_).to(dev)
        coef, ade = self._coef_tensors(self._eps_r, self._sigma_e, self._debye, self._lorentz)
        self._coef = coef
        self._ade_coef = ade if ade.shape[0] else None
        b, c = physics.cpml_profile(n, self.dx, dt, self.cpml_R0, self.cpml_order)
        self._cpml_b, self._cpml_c = to_dev(b if n else np.zeros(1)), to_dev(c if n else np.zeros(1))
        w = (self._waveform_override if self._waveform_override is not None
             else physics.gaussian_derivative(self.total_steps, dt, self.frequency, self.delay_factor))
        self.waveform = to_dev(w)
        field = lambda: torch.zeros((G, ny, nx, W), **f32)
        self._ez = [field(), field()]
        self._hx = [field(), field()]
        self._hy = [field(), field()]
        nn = max(n, 1)
        self._psi_hy = [torch.zeros((G, ny, 2 * nn, W), **f32) for _ in range(2)]
        self._psi_hx = [torch.zeros((G, 2 * nn, nx, W), **f32) for _ in range(2)]
        self._psi_ezx = [torch.zeros((G, ny, 2 * nn, W), **f32) for _ in range(2)]
        self._psi_ezy = [torch.zeros((G, 2 * nn, nx, W), **f32) for _ in range(2)]
        nd, nl = len(self._debye), len(self._lorentz)
        self._j = [torch.zeros((G, nd + nl, ny, nx, W), **f32) for _ in range(2)] if nd + nl else None
        self._j_prev = [torch.zeros((G, nl, ny, nx, W), **f32) for _ in range(2)] if nl else None
        self._status = torch.zeros(1, dtype=torch.int32, device=dev)
        P = len(self.probe_positions)
        self._src = to_dev(np.array(self.source_positions, np.int32).reshape(-1, 2), torch.int32)
        self._prb = to_dev(np.array(self.probe_positions, np.int32).reshape(-1, 2), torch.int32)
        flags = np.zeros(ny, np.uint8)
        for _, y in self.source_positions:
            flags[y] |= 1
        for _, y in self.probe_positions:
            flags[y] |= 2
        self._flags = to_dev(flags, torch.uint8)
        self.probe_data = torch.zeros((B, max(P, 1), self.total_steps), **f32)

        d = Desc2D()
        d.nx, d.ny, d.cpml, d.ntx, d.ntx_pad = nx, ny, n, B, BP
        d.nprobe, d.nsteps, d.n_debye, d.n_lorentz = P, self.total_steps, nd, nl
        d.db, d.inv_dx, d.dt = dt / MU_0, 1.0 / self.dx, dt
        for k in range(2):
            d.ez[k], d.hx[k], d.hy[k] = _ptr(self._ez[k]), _ptr(self._hx[k]), _ptr(self._hy[k])
            d.psi_hy[k], d.psi_hx[k] = _ptr(self._psi_hy[k]), _ptr(self._psi_hx[k])
        for k in range(2):
            d.psi_ezx[k], d.psi_ezy[k] = _ptr(self._psi_ezx[k]), _ptr(self._psi_ezy[k])
            d.j[k] = _ptr(self._j[k]) if self._j is not None else None
            d.j_prev[k] = _ptr(self._j_prev[k]) if self._j_prev is not None else None
        d.coef, d.ade_coef = _ptr(self._coef), _ptr(self._ade_coef)
        d.cpml_b, d.cpml_c = _ptr(self._cpml_b), _ptr(self._cpml_c)
        d.src_xy, d.prb_xy, d.row_flags = _ptr(self._src), _ptr(self._prb), _ptr(self._flags)
        d.waveform, d.probes = _ptr(self.waveform), _ptr(self.probe_data)
        d.status = _ptr(self._status)
        d.rows_per_block = self.rows_per_block
        self._desc = d
        plan = C.c_void_p()
        check(lib().ceep2d_plan_create(C.byref(d), C.byref(plan)), "ceep2d_plan_create")
        self._plan = plan
        self._apply_plan_settings()
        self._built = True

    def _apply_plan_settings(self):
        h, plan = lib(), self._plan
        check(h.ceep2d_plan_set_temporal_block(plan, self.temporal_block), "ceep2d_plan_set_temporal_block")
        check(h.ceep2d_plan_set_frame_split(plan, int(self.frame_split)), "ceep2d_plan_set_frame_split")
        check(h.ceep2d_plan_set_sentinel(plan, self.sentinel_interval), "ceep2d_plan_set_sentinel")
        check(h.ceep2d_plan_set_wait_limit(plan, self.wait_limit_ns), "ceep2d_plan_set_wait_limit")

    def __del__(self):
        if getattr(self, "_plan", None) is not None:
            try:
                lib().ceep2d_plan_destroy(self._plan)
            except Exception:
                pass
            self._plan = None

    def set_rows_per_block(self, rows: int) -> None:
        """Rebuild the launch plan with a given tile height (0 = automatic);
        buffers and state are kept, the state restarts from zero."""
        self.rows_per_block = int(rows)
        if not self._built:
            return
        lib().ceep2d_plan_destroy(self._plan)
        self._plan = None
        self._desc.rows_per_block = self.rows_per_block
        plan = C.c_void_p()
        check(lib().ceep2d_plan_create(C.byref(self._desc), C.byref(plan)), "ceep2d_plan_create")
        self._plan = plan
        self._apply_plan_settings()
        self.reset()

    def autotune(self, candidates=(6, 8, 10, 12, 14, 16), steps: int = 100) -> Dict[int, float]:
        """Pick the tile height (rows per block) by timing `steps` graph-
        replayed steps for each candidate on this solver's grid (two passes,
        the faster of each), and keep the fastest; returns ms per step for
        each.  The results do not depend on
        the tile height (the same cells, the same arithmetic); the state is
        reset afterwards.  Not in the reference: a plan-time choice of this
        framework's launch geometry."""
        if not self._built:
            self._build()
        stream = torch.cuda.current_stream(self.device)
        nst = min(int(steps), self.total_steps)
        if self.temporal_block == 2 and nst > 1:
            nst -= nst % 2
        timings = {}
        for _ in range(2):  # two passes over the candidates, the faster time of each kept
            for rows in candidates:
                self.set_rows_per_block(int(rows))
                self.advance(0, nst, stream=stream)          # capture + warm
                self.reset()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                self.advance(0, nst, stream=stream)
                b.record(stream)
                torch.cuda.synchronize(self.device)
                ms = a.elapsed_time(b) / nst
                timings[int(rows)] = min(ms, timings.get(int(rows), ms))
        best = min(timings, key=timings.get)
        self.set_rows_per_block(best)
        self.reset()
        return timings

    def set_temporal_block(self, steps: int) -> None:
        """Steps per kernel launch: 1, or 2 (two steps per launch, each state
        word read and written once per pair; same arithmetic as 1)."""
        if steps not in (1, 2):
            raise ValueError("temporal block must be 1 or 2 steps")
        self.temporal_block = int(steps)
        if self._built:
            check(lib().ceep2d_plan_set_temporal_block(self._plan, self.temporal_block),
                  "ceep2d_plan_set_temporal_block")

    def set_frame_split(self, on: bool) -> None:
        """Two steps per launch as two kernels: the frame tiles on a side
        stream beside an interior-tile kernel that runs four blocks per SM
        (False, the default: one kernel for every tile).  Bit-identical
        results; faster only where the interior tiles form several waves
        (768^2 x 16 at 12-row tiles: 43.1 against 44.5 us per step)."""
        self.frame_split = bool(on)
        if self._built:
            check(lib().ceep2d_plan_set_frame_split(self._plan, int(self.frame_split)), "ceep2d_plan_set_frame_split")

    def set_sentinel(self, interval: int) -> None:
        """NaN/Inf sentinel: scan Ez and the new probe samples every
        `interval` steps as well as after every run range (0, the default:
        only after every run range).  A hit makes ``run()`` raise."""
        if interval < 0:
            raise ValueError("sentinel interval must be >= 0")
        self.sentinel_interval = int(interval)
        if self._built:
            check(lib().ceep2d_plan_set_sentinel(self._plan, self.sentinel_interval), "ceep2d_plan_set_sentinel")

    def set_wait_limit(self, ns: int) -> None:
        """Bound of the step kernels' device waits in ns (default 1 s)."""
        if ns <= 0:
            raise ValueError("wait limit must be positive")
        self.wait_limit_ns = int(ns)
        if self._built:
            check(lib().ceep2d_plan_set_wait_limit(self._plan, self.wait_limit_ns), "ceep2d_plan_set_wait_limit")

    def inject_copy_fault(self, row: int) -> None:
        """Failure injection for tests: the step kernels copy nothing for grid
        row `row`, so their bounded waits run out (-1 turns it off).  The
        state afterwards is not a simulation state; use a fresh solver."""
        if not self._built:
            self._build()
        check(lib().ceep2d_plan_inject_copy_fault(self._plan, int(row)), "ceep2d_plan_inject_copy_fault")

    def launches(self, nsteps: Optional[int] = None) -> int:
        """Kernel launches that advancing `nsteps` steps (default: all) issues."""
        nsteps = self.total_steps if nsteps is None else int(nsteps)
        if not self._built:
            return nsteps if self.temporal_block == 1 else (nsteps + 1) // 2
        return int(lib().ceep2d_plan_launches(self._plan, nsteps))

    @property
    def plan_rows(self) -> int:
        return lib().ceep2d_plan_rows(self._plan) if self._built else 0

    # -- time loop ------------------------------------------------------------
    def advance(self, step0: int = 0, nsteps: Optional[int] = None, stream=None) -> None:
        """Launch steps [step0, step0+nsteps) on ``stream`` without synchronising."""
        if not self._built:
            self._build()
        nsteps = self.total_steps - step0 if nsteps is None else nsteps
        s = torch.cuda.current_stream(self.device) if stream is None else stream
        check(lib().ceep2d_plan_run(self._plan, step0, nsteps, C.c_void_p(s.cuda_stream),
                                    int(self.use_graph)), "ceep2d_plan_run")

    def run(self) -> Dict[int, Dict[int, np.ndarray]]:
        """All time steps; returns ``{tx: {rx: float64 series of total_steps}}``
        (fdtd_2d_batched.py:408-538).  As in the reference, fields persist, so
        a second call continues the simulation and overwrites the series.
        Leaves ``run_record`` (see ``ceep_b200.trace``)."""
        t0 = time.perf_counter()
        with trace.phase("time_loop"):
            self.advance(0, self.total_steps)
            probe_np = self.probe_data.double().cpu().numpy()
        code = int(self._status.item())
        trace.emit(self, trace.make_record("BatchedFDTD2D", self.nx * self.ny, self.total_steps, self.batch,
                                           time.perf_counter() - t0, code))
        self.check_status(code)
        P = len(self.probe_positions)
        return {tx: {rx: probe_np[tx, rx, :] for rx in range(P)} for tx in range(self.batch)}

    def run_cpu(self) -> Dict[int, Dict[int, np.ndarray]]:
        """The reference's CPML-free variant (fdtd_2d_batched.py:540-611): no
        CPML, fresh fields, H zeroed on the far edge, E on all edges.  In this
        framework it runs on the GPU (a CPML thickness of 0 gives exactly that
        region map); it does not touch this solver's state."""
        twin = BatchedFDTD2D(self.nx, self.ny, self.dx, self.total_steps, 0, self.source_positions,
                             self.probe_positions, self.frequency, self.delay_factor,
                             courant=None if self.dt == self.dx / (C_0 * np.sqrt(2.0)) * 0.99 else self.dt * C_0 / self.dx,
                             waveform=self._waveform_override, device=str(self.device), use_graph=self.use_graph)
        twin._eps_r[:] = self._eps_r
        twin._sigma_e[:] = self._sigma_e
        return twin.run()

    # -- S-parameters (dft.py:55-103, s_params.py:70-137) ---------------------
    def s_matrix(self, frequencies: Optional[Sequence[float]] = None) -> np.ndarray:
        """Complex S[f, rx, tx] = sum_n probe[tx, rx, n] e^{-j w n dt} dt of the
        last run, computed on the device."""
        freqs = self.frequencies if frequencies is None else np.asarray(frequencies, np.float64)
        if freqs is None:
            raise ValueError("no frequencies given")
        from .spectral import dft
        with trace.phase("dft"):
            return dft(self.probe_data[:, :len(self.probe_positions)], freqs,
                       self.dt).cpu().numpy().astype(np.complex128)

    # -- state views in the reference layout (B, nx, ny) ----------------------
    def _cur(self) -> int:
        return lib().ceep2d_plan_current_buffer(self._plan) if self._built else 0

    def _ref_view(self, t: torch.Tensor) -> torch.Tensor:
        """(G, ny, nx, W) device array -> (B, nx, ny) in the reference's axis order."""
        G, ny, nx, W = t.shape
        v = t.permute(0, 3, 2, 1)                       # (G, W, nx, ny)
        v = v.reshape(G * W, nx, ny) if G > 1 else v[0]
        return v[:self.batch]

    @property
    def ez(self):
        return self._ref_view(self._ez[self._cur()]) if self._built else None

    @property
    def hx(self):
        return self._ref_view(self._hx[self._cur()]) if self._built else None

    @property
    def hy(self):
        return self._ref_view(self._hy[self._cur()]) if self._built else None

    def check_status(self, code: Optional[int] = None) -> None:
        """Raise if a bounded device wait gave up, or the NaN/Inf sentinel
        found a non-finite value, during an earlier launch (`code`: the
        status word when the caller has just read it)."""
        if self._built:
            code = int(self._status.item()) if code is None else int(code)
            if code:
                self._status.zero_()
                raise FDTDStatusError(code)

    def reset(self) -> None:
        """Zero every field, psi and ADE state (not in the reference: lets one
        solver be reused for a new phantom without reallocating)."""
        if not self._built:
            return
        for t in (self._ez + self._hx + self._hy + self._psi_hy + self._psi_hx + self._psi_ezx + self._psi_ezy +
                  (self._j or []) + (self._j_prev or []) + [self.probe_data]):
            if t is not None:
                t.zero_()
        check(lib().ceep2d_plan_reset(self._plan), "ceep2d_plan_reset")

    def _coef_tensors(self, eps_r, sigma_e, debye=(), lorentz=()):
        """(nx, ny) FP64 maps -> device (ny, nx, 4) float32 (ca, cb, dt/(eps_r eps0), 0)
        and (poles, ny, nx, 4) ADE coefficients, in the kernel's (y, x) order;
        FP64 arithmetic on the device, bit-identical to the host formulas
        (fdtd_2d_batched.py:151-167, dispersive.py:240-339), in one library
        kernel (physics.coefficient_tensors is the same formula as torch ops)."""
        return physics.coefficient_tensors_kernel(eps_r, sigma_e, self.dt, debye, lorentz, self.device)

    def material_tensors(self, eps_r, sigma_e, debye=(), lorentz=()):
        """Device tensors (coef, ade_coef) for the given (nx, ny) maps in this
        solver's layout, for ``load_material_tensors``."""
        coef, ade = self._coef_tensors(eps_r, sigma_e, debye, lorentz)
        return coef, (ade if ade.shape[0] else None)

    def load_material_tensors(self, mats) -> None:
        """Device-to-device copy of precomputed material tensors into the plan's
        buffers (no host traffic); the pole count must match the first build."""
        if not self._built:
            self._build()
        coef, ade_t = mats
        if (ade_t is None) != (self._ade_coef is None):
            raise ValueError("ADE pole count differs from the built solver")
        self._coef.copy_(coef, non_blocking=True)
        if ade_t is not None:
            self._ade_coef.copy_(ade_t, non_blocking=True)

    def update_materials(self) -> None:
        """Re-upload the coefficients after editing ``_eps_r``/``_sigma_e`` or the
        poles on a built solver."""
        if not self._built:
            return
        coef, ade = self._coef_tensors(self._eps_r, self._sigma_e, self._debye, self._lorentz)
        if ade.shape[0] != (0 if self._ade_coef is None else self._ade_coef.shape[0]):
            raise ValueError("the number of ADE poles cannot change after the first run()")
        self._coef.copy_(coef)
        if ade.shape[0]:
            self._ade_coef.copy_(ade)
