"""CPU oracle for DFT / S-matrix / DAS — TEST INFRASTRUCTURE ONLY.

* ``running_dft``  restates ``DFTMonitor.update`` (src/ceep/solvers/dft.py:55-90):
  re += cos(w n dt) E dt,  im += -sin(w n dt) E dt, with n the step index.
* S layout follows ``MultistaticSParameters`` (src/ceep/solvers/s_params.py:77-79,
  :113-137): ``s_matrix[f, rx, tx]``.
* ``das_frequency`` restates ``DelayAndSumBeamformer._reconstruct_das``
  (src/ceep/imaging/beamforming.py:146-257): pixel (i, j) sits at
  ((x0+i) dx, (y0+j) dx), antennas at grid index * dx, v = C0/sqrt(eps_bg),
  I = |sum_tx sum_rx sum_f S[f,rx,tx] exp(-j 2 pi f (d_tx+d_rx)/v)| including
  tx == rx, then (I - min) / max.
* ``dmas_frequency`` restates ``_reconstruct_dmas`` (beamforming.py:259-313).
* ``das_time`` restates ``das_imaging`` (scripts/verify_dataset_with_das.py:37-103):
  skip tx == rx, idx = int(((|a_tx - p| + |a_rx - p|)/C)/dt) with dt = 1/(4 f),
  pixel += |s[tx, rx, idx]| when 0 <= idx < n_time.
"""
from __future__ import annotations

import numpy as np

from .fdtd2d import C_0


def running_dft(series, dt, frequencies):
    """series: (B, P, T) probe data -> S (F, P, B) complex128, S[f, rx, tx]."""
    series = np.asarray(series, np.float64)
    omega = 2.0 * np.pi * np.asarray(frequencies, np.float64)
    F = omega.size
    B, P, T = series.shape
    re = np.zeros((F, B, P))
    im = np.zeros((F, B, P))
    for step in range(T):
        time = step * dt
        c = np.cos(omega * time).reshape(F, 1, 1)
        s = (-np.sin(omega * time)).reshape(F, 1, 1)
        fld = series[:, :, step]
        re += c * fld * dt
        im += s * fld * dt
    return (re + 1j * im).transpose(0, 2, 1)


def _dist(ax, ay, px, py):
    return np.sqrt((px - ax) ** 2 + (py - ay) ** 2)


def das_frequency(s_matrix, frequencies, antenna_positions, x_range, y_range, dx,
                  background_permittivity=1.0, frequency_range=None, normalize=True):
    s_matrix = np.asarray(s_matrix)
    freqs = np.asarray(frequencies, np.float64)
    if frequency_range is None:
        mask = np.ones(freqs.size, bool)
    else:
        mask = (freqs >= frequency_range[0]) & (freqs <= frequency_range[1])
    f = freqs[mask]
    S = s_matrix[mask]                      # (F, rx, tx)
    v = C_0 / np.sqrt(background_permittivity)
    # ranges are grid indices in the reference (ImagingRegion); a fractional
    # start (an image whose pitch does not divide its origin) is allowed here
    nx = int(round(x_range[1] - x_range[0]))
    ny = int(round(y_range[1] - y_range[0]))
    px = (x_range[0] + np.arange(nx)) * dx
    py = (y_range[0] + np.arange(ny)) * dx
    PX, PY = np.meshgrid(px, py, indexing="ij")
    ant = np.asarray(antenna_positions, np.float64)[:, :2] * dx
    d = np.stack([_dist(a[0], a[1], PX, PY) for a in ant])   # (N, nx, ny)
    image = np.zeros((nx, ny), complex)
    for tx in range(len(ant)):
        for rx in range(len(ant)):
            delay = (d[tx] + d[rx]) / v
            ph = np.exp(-1j * 2 * np.pi * f[:, None, None] * delay[None])
            image += np.sum(S[:, rx, tx][:, None, None] * ph, axis=0)
    return _normalize(np.abs(image), normalize)


def dmas_frequency(s_matrix, frequencies, antenna_positions, x_range, y_range, dx,
                   background_permittivity=1.0, normalize=True):
    s_matrix = np.asarray(s_matrix)
    f = np.asarray(frequencies, np.float64)
    v = C_0 / np.sqrt(background_permittivity)
    nx = x_range[1] - x_range[0]
    ny = y_range[1] - y_range[0]
    px = (x_range[0] + np.arange(nx)) * dx
    py = (y_range[0] + np.arange(ny)) * dx
    PX, PY = np.meshgrid(px, py, indexing="ij")
    ant = np.asarray(antenna_positions, np.float64)[:, :2] * dx
    d = np.stack([_dist(a[0], a[1], PX, PY) for a in ant])
    sig = []
    for tx in range(len(ant)):
        for rx in range(len(ant)):
            delay = (d[tx] + d[rx]) / v
            ph = np.exp(-1j * 2 * np.pi * f[:, None, None] * delay[None])
            sig.append(np.sum(s_matrix[:, rx, tx][:, None, None] * ph, axis=0))
    sig = np.stack(sig)                      # (K, nx, ny)
    total = np.sum(sig, axis=0)
    # sum_{k1<k2} s_k1 conj(s_k2) = (|sum s|^2 - sum |s|^2)/2 only for the real
    # part; compute it directly to keep the imaginary part.
    acc = np.zeros((nx, ny), complex)
    csum = np.conj(total)
    for k in range(sig.shape[0]):
        csum = csum - np.conj(sig[k])
        acc += sig[k] * csum
    return _normalize(np.abs(acc), normalize)


def _normalize(img, normalize):
    if normalize:
        img = img - np.min(img)
        m = np.max(img)
        if m > 0:
            img = img / m
    return img


def das_time(s_matrix, antenna_positions_m, frequency, grid_size, dx):
    """s_matrix (N, N, T) indexed [tx, rx, t]; antenna positions in metres."""
    s_matrix = np.asarray(s_matrix)
    n_ant, _, n_time = s_matrix.shape
    dt = 1 / (4 * frequency)
    C = 3e8
    ant = np.asarray(antenna_positions_m, np.float64)
    image = np.zeros((grid_size, grid_size))
    g = np.arange(grid_size) * dx
    for i in range(grid_size):
        for j in range(grid_size):
            p = np.array([g[i], g[j]])
            acc = 0.0
            for tx in range(n_ant):
                for rx in range(n_ant):
                    if tx == rx:
                        continue
                    dist = np.linalg.norm(ant[tx] - p) + np.linalg.norm(ant[rx] - p)
                    idx = int((dist / C) / dt)
                    if 0 <= idx < n_time:
                        acc += np.abs(s_matrix[tx, rx, idx])
            image[i, j] = acc
    return image
