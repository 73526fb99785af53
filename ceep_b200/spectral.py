"""S-parameters and delay-and-sum imaging on the device.

* ``dft``                  — S[f, rx, tx] from probe series (dft.py:55-90 over
                             every pair, s_params.py:77-79 layout)
* ``MultistaticSParameters`` — the reference container (s_params.py:70-231)
* ``ImagingRegion``, ``DelayAndSumBeamformer`` — beamforming.py:42-313 with the
  DAS and DMAS sums evaluated by CUDA kernels
* ``das_time``             — scripts/verify_dataset_with_das.py:37-103 on the device
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import physics, trace
from ._lib import check, lib
from .constants import C_0


def _stream(device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


_TWIDDLES = {}  # (frequencies, T, dt, device) -> device (F, T, 2) float32; a few entries


def _twiddles(frequencies, T: int, dt: float, device) -> torch.Tensor:
    """The running-DFT weights on the device, built once per (frequencies, T,
    dt): repeated S computations of a dataset reuse them."""
    f = np.ascontiguousarray(np.asarray(frequencies, np.float64))
    key = (f.tobytes(), int(T), float(dt), str(device))
    tw = _TWIDDLES.get(key)
    if tw is None:
        if len(_TWIDDLES) >= 8:
            _TWIDDLES.pop(next(iter(_TWIDDLES)))
        tw = torch.as_tensor(physics.dft_twiddles(f, T, dt)).to(device)
        _TWIDDLES[key] = tw
    return tw


def dft(series: torch.Tensor, frequencies: Sequence[float], dt: float) -> torch.Tensor:
    """series (ntx, nprobe, T) float32 CUDA tensor -> (F, nprobe, ntx) complex64."""
    if not series.is_cuda:
        raise ValueError("series must be a CUDA tensor")
    series = series.contiguous().float()
    B, P, T = series.shape
    tw = _twiddles(frequencies, T, dt, series.device)
    out = torch.empty((len(frequencies), P, B, 2), dtype=torch.float32, device=series.device)
    check(lib().ceep_dft(series.data_ptr(), tw.data_ptr(), out.data_ptr(), B, P, T, len(frequencies),
                         _stream(series.device)), "ceep_dft")
    return torch.view_as_complex(out)


@dataclass
class MultistaticSParameters:
    """s_matrix[f, rx, tx] container with the reference's accessors (s_params.py:70-231)."""
    frequencies: np.ndarray
    s_matrix: np.ndarray
    antenna_positions: List[Tuple[int, ...]]
    background_subtracted: bool = False

    @property
    def num_frequencies(self) -> int:
        return len(self.frequencies)

    @property
    def num_antennas(self) -> int:
        return self.s_matrix.shape[1]

    def get_element(self, tx: int, rx: int, freq_index: Optional[int] = None):
        if freq_index is None:
            return self.s_matrix[:, rx, tx]
        return self.s_matrix[freq_index, rx, tx]

    def get_monostatic(self, freq_index: Optional[int] = None):
        if freq_index is None:
            return np.array([np.diag(self.s_matrix[f]) for f in range(self.num_frequencies)])
        return np.diag(self.s_matrix[freq_index])

    def get_bistatic(self, exclude_monostatic: bool = True):
        out = []
        for tx in range(self.num_antennas):
            for rx in range(self.num_antennas):
                if exclude_monostatic and tx == rx:
                    continue
                out.append((tx, rx, self.s_matrix[:, rx, tx]))
        return out

    def to_db(self) -> "MultistaticSParameters":
        return MultistaticSParameters(self.frequencies, 20 * np.log10(np.abs(self.s_matrix) + 1e-20),
                                      self.antenna_positions, self.background_subtracted)

    def subtract_background(self, background: "MultistaticSParameters") -> "MultistaticSParameters":
        """s_params.py:202-231; with a device tensor on either side the
        difference is formed on that device."""
        if not np.array_equal(self.frequencies, background.frequencies):
            raise ValueError("Frequency points must match")
        a, b = self.s_matrix, background.s_matrix
        if isinstance(a, torch.Tensor) or isinstance(b, torch.Tensor):
            dev = a.device if isinstance(a, torch.Tensor) else b.device
            a, b = torch.as_tensor(a).to(dev), torch.as_tensor(b).to(dev)
        return MultistaticSParameters(self.frequencies, a - b, self.antenna_positions, True)


@dataclass
class ImagingRegion:
    """beamforming.py:42-83."""
    x_range: Tuple[int, int]
    y_range: Tuple[int, int]
    z_slice: Optional[int] = None
    dx: float = 1e-3
    background_permittivity: float = 1.0

    @property
    def nx(self) -> int:
        return self.x_range[1] - self.x_range[0]

    @property
    def ny(self) -> int:
        return self.y_range[1] - self.y_range[0]

    def get_pixel_position(self, i: int, j: int):
        return (self.x_range[0] + i) * self.dx, (self.y_range[0] + j) * self.dx


def das_image(S: torch.Tensor, frequencies: Sequence[float], antenna_xy_m: np.ndarray, nx_pix: int, ny_pix: int,
              px0: float, py0: float, pix: float, velocity: float, normalize: bool = True,
              workspace: Optional[torch.Tensor] = None) -> torch.Tensor:
    """|sum_tx sum_rx sum_f S[f,rx,tx] exp(-j 2 pi f (d_tx + d_rx)/v)| on the device.

    S: (F, N, N) complex64 CUDA tensor, already frequency-masked."""
    dev = S.device
    F, N, _ = S.shape
    Sr = torch.view_as_real(S.to(torch.complex64).contiguous())
    k = torch.as_tensor((2.0 * np.pi * np.asarray(frequencies, np.float64) / velocity).astype(np.float32)).to(dev)
    ant = torch.as_tensor(np.asarray(antenna_xy_m, np.float32).reshape(N, 2)).to(dev)
    need = lib().ceep_das_workspace_bytes(nx_pix, ny_pix, F)
    if need <= 0:
        raise ValueError(f"DAS image {nx_pix}x{ny_pix} x {F} frequencies is not supported")
    if workspace is None or workspace.numel() * workspace.element_size() < need:
        workspace = torch.empty(max(need, 8), dtype=torch.uint8, device=dev)
    img = torch.empty((nx_pix, ny_pix), dtype=torch.float32, device=dev)
    with trace.phase("das"):
        check(lib().ceep_das(Sr.data_ptr(), k.data_ptr(), ant.data_ptr(), F, N, nx_pix, ny_pix, px0, py0, pix,
                             int(normalize), workspace.data_ptr(), img.data_ptr(), _stream(dev)), "ceep_das")
    return img


def dmas_image(S: torch.Tensor, frequencies: Sequence[float], antenna_xy_m: np.ndarray, nx_pix: int, ny_pix: int,
               px0: float, py0: float, pix: float, velocity: float, normalize: bool = True,
               workspace: Optional[torch.Tensor] = None) -> torch.Tensor:
    """|sum_{k1<k2} s_k1 conj(s_k2)| over the delayed pair signals
    s_k = sum_f S[f, rx, tx] exp(-j 2 pi f (d_tx + d_rx)/v), k = tx*N + rx, on
    the device (beamforming.py:259-313).  S: (F, N, N) complex CUDA tensor,
    already frequency-masked."""
    dev = S.device
    F, N, _ = S.shape
    Sr = torch.view_as_real(S.to(torch.complex64).contiguous())
    k = torch.as_tensor((2.0 * np.pi * np.asarray(frequencies, np.float64) / velocity).astype(np.float32)).to(dev)
    ant = torch.as_tensor(np.asarray(antenna_xy_m, np.float32).reshape(N, 2)).to(dev)
    need = lib().ceep_dmas_workspace_bytes(nx_pix, ny_pix)
    if workspace is None or workspace.numel() * workspace.element_size() < need:
        workspace = torch.empty(max(need, 8), dtype=torch.uint8, device=dev)
    img = torch.empty((nx_pix, ny_pix), dtype=torch.float32, device=dev)
    check(lib().ceep_dmas(Sr.data_ptr(), k.data_ptr(), ant.data_ptr(), F, N, nx_pix, ny_pix, px0, py0, pix,
                          int(normalize), workspace.data_ptr(), img.data_ptr(), _stream(dev)), "ceep_dmas")
    return img


class DelayAndSumBeamformer:
    """beamforming.py:86-313; ``reconstruct('das')`` and ``reconstruct('dmas')`` run on the device."""

    def __init__(self, s_parameters: MultistaticSParameters, antenna_positions, imaging_region: ImagingRegion,
                 frequency_range: Optional[Tuple[float, float]] = None, device: str = "cuda"):
        self.s_params = s_parameters
        self.antenna_positions = antenna_positions
        self.region = imaging_region
        self.dx = imaging_region.dx
        if frequency_range is None:
            self.freq_mask = np.ones(len(s_parameters.frequencies), dtype=bool)
        else:
            f_min, f_max = frequency_range
            self.freq_mask = (s_parameters.frequencies >= f_min) & (s_parameters.frequencies <= f_max)
        self.frequencies = s_parameters.frequencies[self.freq_mask]
        self.num_antennas = len(antenna_positions)
        self.velocity = C_0 / np.sqrt(imaging_region.background_permittivity)
        self.device = torch.device(device)

    def compute_delay(self, tx_pos, rx_pos, pixel_pos) -> float:
        tx = np.asarray(tx_pos[:2], np.float64) * self.dx
        rx = np.asarray(rx_pos[:2], np.float64) * self.dx
        p = np.asarray(pixel_pos, np.float64)
        return (np.hypot(*(p - tx)) + np.hypot(*(p - rx))) / self.velocity

    def reconstruct(self, method: str = "das", normalize: bool = True) -> np.ndarray:
        if method not in ("das", "dmas"):
            raise ValueError(f"Unknown method: {method}")
        S = self.s_params.s_matrix
        S = (S[torch.as_tensor(self.freq_mask)] if isinstance(S, torch.Tensor)
             else np.asarray(S)[self.freq_mask])
        S = torch.as_tensor(S).to(self.device)
        ant = np.asarray([p[:2] for p in self.antenna_positions], np.float64) * self.dx
        r = self.region
        image = das_image if method == "das" else dmas_image
        img = image(S, self.frequencies, ant, r.nx, r.ny, r.x_range[0] * r.dx, r.y_range[0] * r.dx, r.dx,
                    self.velocity, normalize)
        return img.double().cpu().numpy()


def das_time(s: torch.Tensor, antenna_positions_m: np.ndarray, frequency: float, grid_size: int,
             dx: float) -> torch.Tensor:
    """Time-domain DAS image (grid, grid) from s[tx, rx, t] (complex or real CUDA tensor)."""
    dev = s.device
    if not torch.is_complex(s):
        s = s.to(torch.complex64)
    sr = torch.view_as_real(s.to(torch.complex64).contiguous())
    N, _, T = s.shape
    ant = torch.as_tensor(np.asarray(antenna_positions_m, np.float64).reshape(N, 2)).to(dev)
    img = torch.empty((grid_size, grid_size), dtype=torch.float32, device=dev)
    check(lib().ceep_das_time(sr.data_ptr(), ant.data_ptr(), N, T, grid_size, float(dx), float(frequency),
                              img.data_ptr(), _stream(dev)), "ceep_das_time")
    return img
