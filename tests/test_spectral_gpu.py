"""Parity of the device DFT and DAS kernels with the reference's own code."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import spectral as osp

pytestmark = pytest.mark.gpu
TOL = 1e-4


def test_dft_against_reference_monitor(cuda_device):
    from ceep_b200 import dft
    g = load_golden("dft_cfg1")
    c = load_golden("fdtd2d_cfg1_float64")
    series = torch.as_tensor(c["probes"], dtype=torch.float32, device=cuda_device)
    S = dft(series, g["frequencies"], float(c["dt"])).cpu().numpy()
    assert S.shape == (101, 8, 8)
    assert rel_l2(S, g["S"]) < TOL


def test_solver_s_matrix_layout(cuda_device):
    """s_matrix()[f, rx, tx] equals the DFT of series[tx][rx] (s_params.py:77-79)."""
    from ceep_b200 import BatchedFDTD2D
    pos_tx = [(20, 20), (40, 25), (30, 44)]
    pos_rx = [(22, 30), (35, 35)]
    s = BatchedFDTD2D(64, 64, 0.5e-3, 300, 8, pos_tx, pos_rx, 2e9, frequencies=np.linspace(0.5e9, 3.5e9, 17))
    out = s.run()
    S = s.s_matrix()
    series = np.array([[out[t][r] for r in range(2)] for t in range(3)])
    ref = osp.running_dft(series, s.dt, s.frequencies)
    assert S.shape == (17, 2, 3)
    assert rel_l2(S, ref) < TOL


@pytest.mark.parametrize("n_ant,nfreq,shape", [(6, 9, (11, 9)), (16, 301, (64, 64)), (3, 1, (5, 7)),
                                               (32, 20, (40, 33)), (9, 50, (1, 1))])
def test_das_against_oracle(cuda_device, n_ant, nfreq, shape):
    from ceep_b200.spectral import das_image
    rng = np.random.default_rng(n_ant * 100 + nfreq)
    f = np.linspace(0.5e9, 3.5e9, nfreq)
    S = (rng.standard_normal((nfreq, n_ant, n_ant)) + 1j * rng.standard_normal((nfreq, n_ant, n_ant)))
    ang = 2 * np.pi * np.arange(n_ant) / n_ant
    pos = [(int(300 + 200 * np.cos(a)), int(300 + 200 * np.sin(a))) for a in ang]
    xr, yr = (268, 268 + shape[0]), (268, 268 + shape[1])
    ref = osp.das_frequency(S, f, pos, xr, yr, 0.5e-3, 4.0)
    img = das_image(torch.as_tensor(S, dtype=torch.complex64, device=cuda_device), f,
                    np.asarray(pos, float) * 0.5e-3, shape[0], shape[1], xr[0] * 0.5e-3, yr[0] * 0.5e-3,
                    0.5e-3, 299_792_458.0 / 2.0).cpu().numpy()
    if shape == (1, 1):
        assert img[0, 0] == 0.0 and ref[0, 0] == 0.0
    else:
        assert rel_l2(img, ref) < TOL


def test_das_against_reference_beamformer(cuda_device):
    from ceep_b200 import DelayAndSumBeamformer, ImagingRegion, MultistaticSParameters
    g = load_golden("das_small")
    pos = [tuple(int(v) for v in p) for p in g["positions"]]
    sp = MultistaticSParameters(g["frequencies"], g["S"], pos)
    region = ImagingRegion(tuple(g["x_range"]), tuple(g["y_range"]), dx=float(g["dx"]),
                           background_permittivity=float(g["eps_bg"]))
    img = DelayAndSumBeamformer(sp, pos, region, frequency_range=tuple(g["frange"])).reconstruct("das")
    assert rel_l2(img, g["das"]) < TOL
    dmas = DelayAndSumBeamformer(sp, pos, region).reconstruct("dmas")
    assert rel_l2(dmas, g["dmas"]) < TOL


@pytest.mark.parametrize("n_ant,nfreq,shape", [(6, 9, (11, 9)), (16, 101, (24, 20)), (3, 1, (5, 7)),
                                               (32, 20, (12, 10)), (9, 50, (1, 1)), (1, 5, (4, 4))])
def test_dmas_against_oracle(cuda_device, n_ant, nfreq, shape):
    from ceep_b200.spectral import dmas_image
    rng = np.random.default_rng(n_ant * 7 + nfreq)
    f = np.linspace(0.5e9, 3.5e9, nfreq)
    S = (rng.standard_normal((nfreq, n_ant, n_ant)) + 1j * rng.standard_normal((nfreq, n_ant, n_ant)))
    ang = 2 * np.pi * np.arange(n_ant) / n_ant
    pos = [(int(300 + 200 * np.cos(a)), int(300 + 200 * np.sin(a))) for a in ang]
    xr, yr = (268, 268 + shape[0]), (268, 268 + shape[1])
    ref = osp.dmas_frequency(S, f, pos, xr, yr, 0.5e-3, 4.0)
    img = dmas_image(torch.as_tensor(S, dtype=torch.complex64, device=cuda_device), f,
                     np.asarray(pos, float) * 0.5e-3, shape[0], shape[1], xr[0] * 0.5e-3, yr[0] * 0.5e-3,
                     0.5e-3, 299_792_458.0 / 2.0).cpu().numpy()
    if shape == (1, 1) or n_ant == 1:
        assert np.all(img == 0.0) and np.all(ref == 0.0)
    else:
        assert rel_l2(img, ref) < TOL


def test_subtract_background_on_device(cuda_device):
    from ceep_b200 import MultistaticSParameters
    rng = np.random.default_rng(3)
    f = np.linspace(1e9, 2e9, 7)
    a = rng.standard_normal((7, 4, 4)) + 1j * rng.standard_normal((7, 4, 4))
    b = rng.standard_normal((7, 4, 4)) + 1j * rng.standard_normal((7, 4, 4))
    pos = [(0, 0)] * 4
    host = MultistaticSParameters(f, a, pos).subtract_background(MultistaticSParameters(f, b, pos))
    dev = MultistaticSParameters(f, torch.as_tensor(a, device=cuda_device), pos).subtract_background(
        MultistaticSParameters(f, b, pos))
    assert dev.background_subtracted and dev.s_matrix.is_cuda
    np.testing.assert_array_equal(dev.s_matrix.cpu().numpy(), host.s_matrix)


def test_das_time_against_reference(cuda_device):
    from ceep_b200 import das_time
    g = load_golden("das_time_small")
    s = torch.as_tensor(g["s"], dtype=torch.complex64, device=cuda_device)
    img = das_time(s, g["positions"], float(g["frequency"]), int(g["grid_size"]), float(g["dx"])).cpu().numpy()
    np.testing.assert_allclose(img, g["image"], rtol=2e-6, atol=0)


def test_das_time_index_truncation_matches_reference(cuda_device):
    """Grid-aligned geometry where many delays land exactly on sample
    boundaries; the FP64 index must truncate exactly like the reference's int()."""
    from ceep_b200 import das_time
    g = load_golden("das_time_aligned")
    s = torch.as_tensor(g["s"], dtype=torch.complex64, device=cuda_device)
    img = das_time(s, g["positions"], float(g["frequency"]), int(g["grid_size"]), float(g["dx"])).cpu().numpy()
    np.testing.assert_array_equal(img, g["image"].astype(np.float32))
