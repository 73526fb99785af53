"""Device-side coefficient maps (physics.coefficient_tensors*, the library kernel) against the host
NumPy formulas they restate (fdtd_2d_batched.py:151-167,
fdtd_3d_batched.py:281-296, dispersive.py:240-339): bit-identical after the
FP32 rounding, for Debye, two-pole Lorentz, scalar and pole-free inputs."""
import numpy as np
import pytest
import torch

from ceep_b200 import physics
from ceep_b200.phantoms import HeadPhantom2D, HeadPhantom3D, LorentzHeadPhantom2D

DT = 1.1674e-12


def _host_2d(eps, sig, deb, lor):
    nx, ny = np.shape(eps)
    eps_add, ade = physics.ade_coefficients(DT, deb, lor, (nx, ny))
    ca, cb = physics.update_coefficients(eps, sig, DT, eps_add if ade.shape[0] else None)
    dteps = DT / (np.asarray(eps, np.float64) * physics.EPS_0)
    coef = np.stack([ca.T, cb.T, dteps.T, np.zeros((ny, nx))], axis=-1).astype(np.float32)
    return coef, ade.transpose(0, 2, 1, 3).astype(np.float32)


def _host_3d(eps, sig, deb, lor):
    shp = eps.shape
    eps_add, ade = physics.ade_coefficients(DT, deb, lor, shp)
    e = eps * physics.EPS_0 + eps_add
    mu = np.ones(shp) * physics.MU_0
    se = sig * DT / (2.0 * e)
    sm = np.zeros(shp) * DT / (2.0 * mu)
    ca, cb = (1.0 - se) / (1.0 + se), (DT / e) / (1.0 + se)
    da, db = (1.0 - sm) / (1.0 + sm), (DT / mu) / (1.0 + sm)
    coef = np.stack([da, db, ca, cb], -1).transpose(2, 1, 0, 3).astype(np.float32)
    return coef, ade.transpose(0, 3, 2, 1, 4).astype(np.float32)


def _cases_2d():
    for ph in (HeadPhantom2D(120, 110, 0.5e-3, seed=3), LorentzHeadPhantom2D(96, 104, 0.5e-3, seed=4)):
        e, s = ph.get_eps_map()
        d = ph.get_dispersion()
        yield e, s, d["debye"], d["lorentz"]
    yield np.full((5, 7), 3.0), 0.2, [(10.0, 8e-12)], []
    yield np.full((5, 7), 3.0), np.zeros((5, 7)), [], []
    # one Debye and one Lorentz pole per cell, poles absent in part of the grid
    lph = LorentzHeadPhantom2D(64, 72, 0.5e-3, seed=6)
    e, s = lph.get_eps_map()
    lor = lph.get_dispersion()["lorentz"][:1]
    de = np.where(lor[0][0] > 0, 12.0, 0.0)
    yield e, s, [(de, np.where(de > 0, 7e-12, 0.0))], lor


def _check(device):
    for e, s, deb, lor in _cases_2d():
        c0, a0 = _host_2d(e, s, deb, lor)
        c1, a1 = physics.coefficient_tensors(e, s, DT, deb, lor, device)
        assert np.array_equal(c0, c1.cpu().numpy()) and np.array_equal(a0, a1.cpu().numpy())
    ph = HeadPhantom3D(40, 36, 32, 1e-3, seed=5, semi_axes=(0.012, 0.011, 0.01))
    e, s = ph.get_eps_map_3d()
    d = ph.get_dispersion()
    c0, a0 = _host_3d(e, s, d["debye"], d["lorentz"])
    c1, a1 = physics.coefficient_tensors_3d(e, s, np.ones(e.shape), np.zeros(e.shape), DT, d["debye"],
                                            d["lorentz"], device)
    assert np.array_equal(c0, c1.cpu().numpy()) and np.array_equal(a0, a1.cpu().numpy())


def test_coefficient_tensors_cpu():
    _check("cpu")


@pytest.mark.gpu
def test_coefficient_tensors_cuda(cuda_device):
    _check(cuda_device)


@pytest.mark.gpu
def test_coefficient_kernel_cuda(cuda_device):
    """The library's one-pass coefficient kernel (the solver's material path)
    gives the host formulas' FP32 bits as well."""
    for e, s, deb, lor in _cases_2d():
        c0, a0 = _host_2d(e, s, deb, lor)
        c1, a1 = physics.coefficient_tensors_kernel(e, s, DT, deb, lor, cuda_device)
        assert np.array_equal(c0, c1.cpu().numpy()) and np.array_equal(a0, a1.cpu().numpy())
