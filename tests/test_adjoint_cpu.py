"""Gradient oracle pins (CPU): the PyTorch restatement equals the NumPy oracle,
and its autograd gradient equals central finite differences (h = 1e-3) of the
FP64 oracle on 32 random interior cells for eps_r, sigma, Debye delta_eps and
tau (step 1e-3 of the value's scale)."""
import numpy as np
import torch

from oracle.fdtd2d import Fdtd2DOracle
from oracle.spectral import running_dft
from oracle.torch_fdtd2d import TorchFdtd2D, s_misfit_loss

NX, NY, N, T = 36, 32, 4, 110
SRC = [(12, 11), (23, 20)]
PRB = [(12, 11), (23, 20), (18, 26)]
FREQS = np.linspace(1e9, 3e9, 9)


def _maps():
    x, y = np.meshgrid(np.arange(NX), np.arange(NY), indexing="ij")
    m = (x - 18) ** 2 + (y - 16) ** 2 <= 7 ** 2
    return (np.where(m, 6.0, 1.0), np.where(m, 0.4, 0.0), np.where(m, 18.0, 0.0), np.where(m, 8e-12, 0.0), m)


def _oracle_loss(eps, sig, de, tau, target):
    o = Fdtd2DOracle(NX, NY, 0.5e-3, T, N, SRC, PRB, 2e9, eps_r=eps, sigma_e=sig,
                     dispersion={"debye": [(de, tau)]})
    o.run()
    S = running_dft(o.probe_data, o.dt, FREQS)
    return float(np.sum(np.abs(S - target) ** 2)), o


def test_torch_restatement_equals_oracle():
    eps, sig, de, tau, _ = _maps()
    _, o = _oracle_loss(eps, sig, de, tau, 0.0)
    t = TorchFdtd2D(NX, NY, 0.5e-3, T, N, SRC, PRB, 2e9)
    tt = lambda a: torch.as_tensor(a, dtype=torch.float64)
    p = t.run(tt(eps), tt(sig), [(tt(de), tt(tau))]).numpy()
    assert np.abs(p - o.probe_data).max() <= 1e-12 * np.abs(o.probe_data).max()


def test_autograd_matches_central_differences():
    eps, sig, de, tau, m = _maps()
    # target: a different inclusion
    eps_t = eps.copy(); eps_t[15:21, 13:19] = 12.0
    _, ot = _oracle_loss(eps_t, sig, de, tau, 0.0)
    target = running_dft(ot.probe_data, ot.dt, FREQS)
    t = TorchFdtd2D(NX, NY, 0.5e-3, T, N, SRC, PRB, 2e9)
    e_ = torch.tensor(eps, dtype=torch.float64, requires_grad=True)
    s_ = torch.tensor(sig, dtype=torch.float64, requires_grad=True)
    d_ = torch.tensor(de, dtype=torch.float64, requires_grad=True)
    t_ = torch.tensor(tau, dtype=torch.float64, requires_grad=True)
    probes = t.run(e_, s_, [(d_, t_)])
    loss, _ = s_misfit_loss(probes, t.dt, FREQS, torch.as_tensor(target))
    loss.backward()
    rng = np.random.default_rng(3)
    cells = [tuple(c) for c in np.argwhere(m)[rng.choice(int(m.sum()), 32, replace=False)]]
    for name, base, grad, h in (("eps_r", eps, e_.grad, 1e-3), ("sigma", sig, s_.grad, 1e-3),
                                ("deps", de, d_.grad, 1e-3), ("tau", tau, t_.grad, 8e-15)):
        fd, ad = [], []
        for c in cells:
            vals = []
            for sgn in (1, -1):
                arr = base.copy()
                arr[c] += sgn * h
                args = {"eps_r": (arr, sig, de, tau), "sigma": (eps, arr, de, tau), "deps": (eps, sig, arr, tau),
                        "tau": (eps, sig, de, arr)}[name]
                vals.append(_oracle_loss(*args, target)[0])
            fd.append((vals[0] - vals[1]) / (2 * h))
            ad.append(float(grad[c]))
        fd, ad = np.array(fd), np.array(ad)
        err = np.linalg.norm(fd - ad) / np.linalg.norm(fd)
        assert err < 1e-4, (name, err)


def test_segment_schedule_serial():
    """The serial backward schedule: kept segments are read from their own
    buffers, every other segment is recomputed into its buffer just before
    its adjoint reads it, last segment first."""
    from ceep_b200.adjoint import run_segments_backward
    starts = [88, 77, 66, 55, 44, 33]
    for kept in ({88}, {88, 77}, {88, 77, 66}, set(starts)):
        nbuf = max(1, len(kept))
        log, holds = [], {}
        rec = lambda a, b: (log.append(("r", a, b)), holds.__setitem__(b, a))
        adj = lambda a, b: log.append(("a", a, b, holds.get(b)))
        for i, a in enumerate(starts):       # the forward pass left the kept ones in buffer i
            if a in kept:
                holds[i] = a
        run_segments_backward(starts, kept, rec, adj, "cpu", False, nbuf)
        assert [e[1] for e in log if e[0] == "a"] == starts
        assert all(e[3] == e[1] for e in log if e[0] == "a")       # each adjoint reads its own segment
        assert sorted(e[1] for e in log if e[0] == "r") == sorted(set(starts) - kept)


def _lorentz_maps():
    eps, sig, de, tau, m = _maps()
    x, y = np.meshgrid(np.arange(NX), np.arange(NY), indexing="ij")
    ml = (x - 16) ** 2 + (y - 15) ** 2 <= 5 ** 2
    ldeps = np.where(ml, 4.0, 0.0)
    lw0 = np.where(ml, 2 * np.pi * 6e9, 0.0)
    ld = np.where(ml, 2 * np.pi * 0.5e9, 0.0)
    return eps, sig, de, tau, (ldeps, lw0, ld), ml


def _oracle_loss_lor(eps, sig, de, tau, lor, target):
    o = Fdtd2DOracle(NX, NY, 0.5e-3, T, N, SRC, PRB, 2e9, eps_r=eps, sigma_e=sig,
                     dispersion={"debye": [(de, tau)], "lorentz": [lor]})
    o.run()
    S = running_dft(o.probe_data, o.dt, FREQS)
    return float(np.sum(np.abs(S - target) ** 2)), o


def test_torch_restatement_with_a_lorentz_pole_equals_oracle():
    eps, sig, de, tau, lor, _ = _lorentz_maps()
    _, o = _oracle_loss_lor(eps, sig, de, tau, lor, 0.0)
    t = TorchFdtd2D(NX, NY, 0.5e-3, T, N, SRC, PRB, 2e9)
    tt = lambda a: torch.as_tensor(a, dtype=torch.float64)
    p = t.run(tt(eps), tt(sig), [(tt(de), tt(tau))], [tuple(tt(a) for a in lor)]).numpy()
    assert np.abs(p - o.probe_data).max() <= 1e-12 * np.abs(o.probe_data).max()


def test_lorentz_delta_eps_gradient_matches_central_differences():
    """d(S misfit)/d(Lorentz delta_eps) by autograd through the restatement
    against central differences (h = 1e-3) of the FP64 oracle on 12 cells of
    the Lorentz region (omega_0 and delta held fixed)."""
    eps, sig, de, tau, (ldeps, lw0, ld), ml = _lorentz_maps()
    eps_t = eps.copy(); eps_t[15:21, 13:19] = 12.0
    _, ot = _oracle_loss_lor(eps_t, sig, de, tau, (ldeps, lw0, ld), 0.0)
    target = running_dft(ot.probe_data, ot.dt, FREQS)
    t = TorchFdtd2D(NX, NY, 0.5e-3, T, N, SRC, PRB, 2e9)
    tt = lambda a: torch.as_tensor(a, dtype=torch.float64)
    l_ = torch.tensor(ldeps, dtype=torch.float64, requires_grad=True)
    probes = t.run(tt(eps), tt(sig), [(tt(de), tt(tau))], [(l_, tt(lw0), tt(ld))])
    loss, _ = s_misfit_loss(probes, t.dt, FREQS, torch.as_tensor(target))
    loss.backward()
    rng = np.random.default_rng(5)
    cells = [tuple(c) for c in np.argwhere(ml)[rng.choice(int(ml.sum()), 12, replace=False)]]
    fd, ad = [], []
    for c in cells:
        vals = []
        for sgn in (1, -1):
            arr = ldeps.copy()
            arr[c] += sgn * 1e-3
            vals.append(_oracle_loss_lor(eps, sig, de, tau, (arr, lw0, ld), target)[0])
        fd.append((vals[0] - vals[1]) / 2e-3)
        ad.append(float(l_.grad[c]))
    fd, ad = np.array(fd), np.array(ad)
    assert np.linalg.norm(fd - ad) / np.linalg.norm(fd) < 1e-4
