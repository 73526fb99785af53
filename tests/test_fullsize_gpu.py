"""Parity at the benchmarked sizes, against fixtures made in FP64 and FP32 by
the reference's own solver and by the oracle (tests/golden/make_golden.py).

* head600 (the head-imaging sample, 600x600, 16 TX on a ring of radius 200
  cells, 800 steps, CPML 15): the reference's own BatchedFDTD2D.run()
  (src/ceep/solvers/fdtd_2d_batched.py:408-538) in FP32 and FP64 on the
  seeded head phantom's non-dispersive maps; and the oracle in FP64 on the
  same phantom with its Debye pole per layer, through S at 301 frequencies
  (dft.py:55-90) and the 64x64 DAS image (beamforming.py:210-257).
* head192 (192^3, 1 mm, 1000 steps, CPML 10, 8 Ez dipoles, Debye shells with
  an inclusion): the 3D oracle in FP64 (fdtd_3d_batched.py:886-985), four of
  the eight transmit events.

The bar is the north star's 1e-4 relative L2 (over whole arrays: every TX,
probe and step, or every frequency and pair); each test prints the measured
error and, where a reference FP64 run exists, the error against it, which is
the FP32 drift over the full step count.
"""
import hashlib
import os

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu
GOLD = os.path.join(ROOT, "tests", "golden")
TOL = 1e-4


def _load(name):
    path = os.path.join(GOLD, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"{name}.npz not generated")
    return np.load(path)


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(np.asarray(a, np.float64)).tobytes())
    return h.hexdigest()


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _head600(dispersive):
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.phantoms import HeadPhantom2D, ring_positions
    pos = ring_positions(16, (300, 300), 200)
    ph = HeadPhantom2D(600, 600, 0.5e-3, seed=1000)
    eps, sig = ph.get_eps_map()
    (de, tau), = ph.get_dispersion()["debye"]
    freqs = np.linspace(0.5e9, 3.5e9, 301)
    s = BatchedFDTD2D(600, 600, 0.5e-3, 800, 15, pos, pos, 2e9, frequencies=freqs, device="cuda:0")
    if dispersive:
        s.set_phantom(ph)
        sha = _sha(eps, sig, de, tau)
    else:
        s._eps_r[:], s._sigma_e[:] = eps, sig
        sha = _sha(eps, sig)
    s.run()
    return s, pos, freqs, sha


def test_head600_probes_match_the_reference_run_fp32_and_fp64():
    g32, g64 = _load("head600_ref_float32"), _load("head600_ref_float64")
    s, pos, _, sha = _head600(dispersive=False)
    assert str(g32["inputs_sha"]) == sha == str(g64["inputs_sha"]), "phantom generator changed"
    assert np.array_equal(g32["positions"], np.array(pos))
    got = s.probe_data.double().cpu().numpy()
    e32 = rel_l2(got, g32["probes"].astype(np.float64))
    e64 = rel_l2(got, g64["probes"])
    ref_drift = rel_l2(g32["probes"].astype(np.float64), g64["probes"])
    worst = max(rel_l2(got[t], g64["probes"][t]) for t in range(16))
    print(f"head600 probes (16x16x800): vs reference FP32 {e32:.3e}, vs reference FP64 {e64:.3e} "
          f"(worst TX {worst:.3e}); reference FP32 vs FP64 {ref_drift:.3e}")
    assert e32 < TOL and e64 < TOL


def test_head600_debye_probes_s_and_das_match_the_oracle():
    from ceep_b200.spectral import das_image
    g = _load("head600_oracle")
    s, pos, freqs, sha = _head600(dispersive=True)
    assert str(g["inputs_sha"]) == sha, "phantom generator changed"
    got = s.probe_data.double().cpu().numpy()
    e_p = rel_l2(got, g["probes"])
    S = s.s_matrix()
    e_s = rel_l2(S, g["S"])
    npix, half, dx = 64, 0.09, 0.5e-3
    img = das_image(torch.as_tensor(S, dtype=torch.complex64, device="cuda:0"), freqs,
                    np.asarray(pos, float) * dx, npix, npix, 300 * dx - half, 300 * dx - half, 2 * half / npix,
                    299_792_458.0).cpu().numpy()
    e_d = rel_l2(img, g["das"])
    print(f"head600 Debye vs oracle FP64: probes {e_p:.3e}, S (301x16x16) {e_s:.3e}, DAS 64x64 {e_d:.3e}")
    assert e_p < TOL and e_s < TOL and e_d < TOL


def test_head192_probes_and_s_match_the_3d_oracle():
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.phantoms import HeadPhantom3D, ring_positions
    from oracle.spectral import running_dft
    g = _load("head192_oracle")
    pos = [(x, y, 96) for x, y in ring_positions(8, (96, 96), 75)]
    ph = HeadPhantom3D(192, 192, 192, 1e-3, seed=1000)
    eps, sig = ph.get_eps_map_3d()
    (de, tau), = ph.get_dispersion()["debye"]
    assert str(g["inputs_sha"]) == _sha(eps, sig, de, tau), "phantom generator changed"
    freqs = np.linspace(0.5e9, 3.5e9, 101)
    s = BatchedFDTD3D(192, 192, 192, 1e-3, 1000, 10, pos, pos, 2e9, frequencies=freqs, device="cuda:0")
    s.set_phantom(ph)
    s.run()
    tx = [int(t) for t in g["tx"]]
    got = s.probe_data.double().cpu().numpy()[tx]
    e_p = rel_l2(got, g["probes"])
    S_ref = running_dft(g["probes"], float(g["dt"]), freqs)          # (F, rx, 4 TX)
    S = s.s_matrix()[:, :, tx]
    e_s = rel_l2(S, S_ref)
    print(f"head192 (192^3, 1000 steps) vs 3D oracle FP64: probes {e_p:.3e}, S (101x8x4) {e_s:.3e}")
    assert e_p < TOL and e_s < TOL
