"""Edge cases of the batched solvers against the oracle: no probes, one TX,
transmit events sharing a source cell, repeated probe positions, TX counts
just past a padding or group boundary, a one-step run."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle.fdtd2d import Fdtd2DOracle
from oracle.fdtd3d import Fdtd3DOracle

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _maps(nx, ny, seed, nz=None):
    rng = np.random.default_rng(seed)
    shp = (nx, ny) if nz is None else (nx, ny, nz)
    eps = 1.0 + 20.0 * (rng.random(shp) < 0.3) * rng.random(shp)
    return eps, 0.5 * rng.random(shp) * (eps > 1)


def test_2d_without_probes(cuda_device):
    from ceep_b200 import BatchedFDTD2D
    eps, sig = _maps(40, 36, 1)
    s = BatchedFDTD2D(40, 36, 0.5e-3, 80, 5, [(15, 17), (22, 20)], [], 2e9)
    s._eps_r[:], s._sigma_e[:] = eps, sig
    out = s.run()
    assert out == {0: {}, 1: {}}
    o = Fdtd2DOracle(40, 36, 0.5e-3, 80, 5, [(15, 17), (22, 20)], [], 2e9, eps_r=eps, sigma_e=sig)
    o.run()
    assert rel_l2(s.ez.cpu().numpy(), o.ez) < TOL


@pytest.mark.parametrize("ntx", [1, 5, 17, 33, 65])
def test_2d_tx_counts_and_collisions(cuda_device, ntx):
    """TX counts past each padding / group boundary; the first two TX share
    a source cell and the probe list repeats a position, so their series
    must match each other bit for bit."""
    from ceep_b200 import BatchedFDTD2D
    nx, ny, n, T = 44, 40, 5, 90
    rng = np.random.default_rng(ntx)
    src = [(int(rng.integers(n + 1, nx - n - 1)), int(rng.integers(n + 1, ny - n - 1))) for _ in range(ntx)]
    if ntx > 1:
        src[1] = src[0]
    prb = [(10, 10), (30, 25), (10, 10), src[-1]]
    eps, sig = _maps(nx, ny, 100 + ntx)
    s = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, src, prb, 2e9)
    s._eps_r[:], s._sigma_e[:] = eps, sig
    out = s.run()
    got = np.array([[out[b][p] for p in range(len(prb))] for b in range(ntx)])
    o = Fdtd2DOracle(nx, ny, 0.5e-3, T, n, src, prb, 2e9, eps_r=eps, sigma_e=sig)
    o.run()
    assert rel_l2(got, o.probe_data) < TOL
    assert np.array_equal(got[:, 0], got[:, 2])
    if ntx > 1:
        assert np.array_equal(got[0], got[1])


def test_2d_one_step(cuda_device):
    from ceep_b200 import BatchedFDTD2D
    s = BatchedFDTD2D(30, 30, 0.5e-3, 1, 4, [(14, 15)], [(14, 15), (20, 20)], 2e9)
    out = s.run()
    o = Fdtd2DOracle(30, 30, 0.5e-3, 1, 4, [(14, 15)], [(14, 15), (20, 20)], 2e9)
    o.run()
    assert rel_l2(np.array([out[0][0], out[0][1]]), o.probe_data[0]) < TOL


@pytest.mark.parametrize("ntx", [1, 9])
def test_3d_tx_counts_collisions_and_no_probes(cuda_device, ntx):
    from ceep_b200 import BatchedFDTD3D
    nx, ny, nz, n, T = 20, 18, 16, 3, 40
    rng = np.random.default_rng(7 + ntx)
    src = [tuple(int(rng.integers(n + 1, m - n - 1)) for m in (nx, ny, nz)) for _ in range(ntx)]
    if ntx > 1:
        src[1] = src[0]
    prb = [(9, 9, 8), (12, 5, 10), (9, 9, 8)]
    eps, sig = _maps(nx, ny, 40 + ntx, nz)
    s = BatchedFDTD3D(nx, ny, nz, 1e-3, T, n, src, prb, 2e9)
    s._eps_r[:], s._sigma_e[:] = eps, sig
    out = s.run()
    got = np.array([[out[b][p] for p in range(len(prb))] for b in range(ntx)])
    o = Fdtd3DOracle(nx, ny, nz, 1e-3, T, n, src, prb, 2e9, eps_r=eps, sigma_e=sig)
    o.run()
    assert rel_l2(got, o.probe_data) < TOL
    assert np.array_equal(got[:, 0], got[:, 2])
    if ntx > 1:
        assert np.array_equal(got[0], got[1])
    s2 = BatchedFDTD3D(nx, ny, nz, 1e-3, T, n, src, [], 2e9)
    s2._eps_r[:], s2._sigma_e[:] = eps, sig
    assert s2.run() == {b: {} for b in range(ntx)}
    assert torch.equal(s2.ez, s.ez)
