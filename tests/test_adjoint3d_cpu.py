"""3D gradient oracle pins (CPU): the PyTorch restatement (which leaves out the
H-CPML faces, since they cannot reach a probe) equals the full NumPy 3D
oracle, and its autograd gradient equals central finite differences of the
FP64 oracle on random interior cells for eps_r, sigma, Debye delta_eps and
tau."""
import numpy as np
import torch

from oracle.fdtd3d import Fdtd3DOracle
from oracle.torch_fdtd3d import TorchFdtd3D

NX, NY, NZ, N, T = 20, 18, 16, 3, 70
SRC = [(8, 8, 8), (11, 10, 7)]
PRB = [(8, 8, 8), (11, 10, 7), (12, 6, 9), (1, 9, 8)]   # the last one in the CPML shell


def _maps():
    x, y, z = np.meshgrid(np.arange(NX), np.arange(NY), np.arange(NZ), indexing="ij")
    m = (x - 10) ** 2 + (y - 9) ** 2 + (z - 8) ** 2 <= 3.5 ** 2
    rng = np.random.default_rng(11)
    eps = np.where(m, 6.0 + rng.random(m.shape), 1.0)
    sig = np.where(m, 0.4 + 0.1 * rng.random(m.shape), 0.0)
    return eps, sig, np.where(m, 18.0, 0.0), np.where(m, 8e-12, 0.0), m


def _oracle(eps, sig, de, tau):
    o = Fdtd3DOracle(NX, NY, NZ, 1e-3, T, N, SRC, PRB, 2e9, eps_r=eps, sigma_e=sig,
                     dispersion={"debye": [(de, tau)]})
    o.run()
    return o.probe_data


def test_torch_restatement_equals_full_oracle():
    eps, sig, de, tau, _ = _maps()
    ref = _oracle(eps, sig, de, tau)
    tt = lambda a: torch.as_tensor(a, dtype=torch.float64)
    p = TorchFdtd3D(NX, NY, NZ, 1e-3, T, N, SRC, PRB, 2e9).run(tt(eps), tt(sig), [(tt(de), tt(tau))]).numpy()
    assert np.abs(ref).max() > 0
    assert np.abs(p - ref).max() <= 1e-12 * np.abs(ref).max()


def test_autograd_matches_central_differences():
    eps, sig, de, tau, m = _maps()
    G = np.random.default_rng(5).standard_normal((len(SRC), len(PRB), T))
    t = TorchFdtd3D(NX, NY, NZ, 1e-3, T, N, SRC, PRB, 2e9)
    ins = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in (eps, sig, de, tau)]
    loss = (t.run(ins[0], ins[1], [(ins[2], ins[3])]) * torch.as_tensor(G)).sum()
    loss.backward()
    rng = np.random.default_rng(3)
    cells = [tuple(c) for c in np.argwhere(m)[rng.choice(int(m.sum()), 10, replace=False)]]
    base = (eps, sig, de, tau)
    for k, (name, h) in enumerate((("eps_r", 1e-3), ("sigma", 1e-3), ("deps", 1e-3), ("tau", 8e-15))):
        fd, ad = [], []
        for c in cells:
            vals = []
            for sgn in (1, -1):
                args = [a.copy() for a in base]
                args[k][c] += sgn * h
                vals.append(float((_oracle(*args) * G).sum()))
            fd.append((vals[0] - vals[1]) / (2 * h))
            ad.append(float(ins[k].grad[c]))
        fd, ad = np.array(fd), np.array(ad)
        err = np.linalg.norm(fd - ad) / np.linalg.norm(fd)
        assert err < 1e-4, (name, err)
