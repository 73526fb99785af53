"""The CUDA adjoint against autograd through the PyTorch FP64 restatement
(itself pinned to central finite differences of the FP64 oracle on the CPU)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle.torch_fdtd2d import TorchFdtd2D, s_misfit_loss

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _case(nx, ny, n, seed, debye=True, nring=4):
    rng = np.random.default_rng(seed)
    x, y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    cx, cy = nx // 2, ny // 2
    r = min(nx, ny) // 4
    m = (x - cx) ** 2 + (y - cy) ** 2 <= r ** 2
    eps = np.where(m, 6.0 + rng.random((nx, ny)), 1.0)
    sig = np.where(m, 0.3 + 0.2 * rng.random((nx, ny)), 0.0)
    de = np.where(m, 15.0 + 5 * rng.random((nx, ny)), 0.0) if debye else None
    tau = np.where(m, 8e-12, 0.0) if debye else None
    ang = 2 * np.pi * np.arange(nring) / nring
    ring = [(int(cx + (r + 6) * np.cos(a)), int(cy + (r + 6) * np.sin(a))) for a in ang]
    return eps, sig, de, tau, m, ring


def _run_both(nx, ny, n, T, seed, K, debye=True, ntx=3, loss="vjp", nring=4, grad_tau=False):
    """Gradient of the same scalar through the CUDA adjoint and through autograd
    of the FP64 restatement.  loss="vjp": sum(probes * G) for a fixed random G,
    which tests the transposed Jacobian alone; loss="misfit": the S-parameter
    misfit to a well-separated target."""
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.adjoint import Adjoint2D, probes_with_grad, s_parameter_loss
    dev = torch.device("cuda")
    eps, sig, de, tau, m, ring = _case(nx, ny, n, seed, debye, nring)
    src, prb = ring[:ntx], ring
    freqs = np.linspace(1e9, 3e9, 11)
    t = TorchFdtd2D(nx, ny, 0.5e-3, T, n, src, prb, 2e9, device=dev)
    f64 = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    G = torch.as_tensor(np.random.default_rng(seed + 100).standard_normal((ntx, len(prb), T)), device=dev)
    target = None
    if loss == "misfit":
        eps_t = np.where(m, 1.0 + 0.5 * (eps - 1.0), 1.0)          # a clearly different head
        deb_t = [(f64(de), f64(tau))] if debye else []
        with torch.no_grad():
            _, target = s_misfit_loss(t.run(f64(eps_t), f64(sig), deb_t), t.dt, freqs, 0.0)
    scalar = (lambda p, dt: (p * G).sum()) if loss == "vjp" else \
        (lambda p, dt: s_parameter_loss(p, dt, freqs, target)[0])
    e_, s_ = f64(eps).requires_grad_(True), f64(sig).requires_grad_(True)
    d_ = f64(de).requires_grad_(True) if debye else None
    t_ = f64(tau).requires_grad_(grad_tau) if debye else None
    ref = scalar(t.run(e_, s_, [(d_, t_)] if debye else []), t.dt)
    ref.backward()
    s = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, src, prb, 2e9)
    if debye:
        s.set_dispersion(debye=[(de, tau)])
    adj = Adjoint2D(s, checkpoint_every=K, grad_tau=grad_tau)
    e2, s2 = f64(eps).requires_grad_(True), f64(sig).requires_grad_(True)
    d2 = f64(de).requires_grad_(True) if debye else None
    t2 = f64(tau).requires_grad_(grad_tau) if debye else None
    val = scalar(probes_with_grad(e2, s2, adj, d2, t2).double(), s.dt)
    val.backward()
    inner = np.zeros((nx, ny), bool)
    inner[n + 1:nx - n, n + 1:ny - n] = True
    out = {"value": (float(val.detach()), float(ref.detach())), "eps_r": (e2.grad, e_.grad), "sigma": (s2.grad, s_.grad)}
    if debye:
        out["deps"] = (d2.grad, d_.grad)
    if grad_tau:
        out["tau"] = (t2.grad, t_.grad)
    return out, inner


def _check(out, inner, keys, tol):
    for k in keys:
        g, gr = (v.detach().cpu().numpy() for v in out[k])
        err = rel_l2(g[inner], gr[inner])
        print(f"{k}: rel L2 vs autograd {err:.2e}")
        assert err < tol, (k, err)


def test_adjoint_vjp_matches_autograd(cuda_device):
    out, inner = _run_both(96, 88, 8, 220, 1, K=25)
    _check(out, inner, ("eps_r", "sigma", "deps"), TOL)


def test_adjoint_torch_check_128_300(cuda_device):
    out, inner = _run_both(128, 128, 10, 300, 2, K=50, ntx=4)
    _check(out, inner, ("eps_r", "sigma", "deps"), TOL)


def test_adjoint_16tx_interior_blocks(cuda_device):
    """16 TX (four float4 lanes per cell, 32-cell blocks): most blocks lie in
    the plain interior and take the kernel path without region tests."""
    out, inner = _run_both(112, 112, 8, 160, 6, K=20, ntx=16, nring=16)
    _check(out, inner, ("eps_r", "sigma", "deps"), TOL)


def test_adjoint_two_tx_groups(cuda_device):
    """37 TX: two TX groups, whose per-group gradient sums are added."""
    out, inner = _run_both(100, 92, 7, 140, 7, K=1, ntx=37, nring=37)
    _check(out, inner, ("eps_r", "sigma", "deps"), TOL)


def test_adjoint_tau_gradient(cuda_device):
    """grad_tau: the forward keeps J of every step and the adjoint adds the
    k1 and gamma terms, giving d/dtau; the other gradients do not change."""
    for K in (1, 30):
        out, inner = _run_both(96, 88, 8, 200, 8, K=K, grad_tau=True)
        _check(out, inner, ("eps_r", "sigma", "deps", "tau"), TOL)


def test_adjoint_without_dispersion(cuda_device):
    out, inner = _run_both(64, 60, 6, 150, 3, K=10, debye=False)
    _check(out, inner, ("eps_r", "sigma"), TOL)


def test_s_misfit_gradient(cuda_device):
    # the residual S - S* is a difference of FP32-derived spectra, so the
    # bound is looser than for the bare transposed Jacobian above
    out, inner = _run_both(96, 88, 8, 220, 4, K=1, loss="misfit")
    v, vr = out["value"]
    assert abs(v - vr) / vr < 1e-3
    _check(out, inner, ("eps_r", "sigma", "deps"), 1e-3)


def test_checkpoint_interval_does_not_change_the_gradient(cuda_device):
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.adjoint import Adjoint2D, probes_with_grad
    eps, sig, de, tau, m, ring = _case(70, 66, 6, 5)
    res = []
    for K in (1, 7, 40):
        s = BatchedFDTD2D(70, 66, 0.5e-3, 120, 6, ring[:3], ring, 2e9)
        s.set_dispersion(debye=[(de, tau)])
        adj = Adjoint2D(s, checkpoint_every=K)
        e = torch.tensor(eps, dtype=torch.float64, device="cuda", requires_grad=True)
        p = probes_with_grad(e, torch.tensor(sig, device="cuda"), adj, torch.tensor(de, device="cuda"),
                             torch.tensor(tau, device="cuda"))
        (p.double() ** 2).sum().backward()
        res.append(e.grad.clone())
    assert torch.equal(res[0], res[1]) and torch.equal(res[0], res[2])


def test_overlapped_recompute_gives_the_same_gradient(cuda_device):
    """The two-stream backward (recompute of the next segment beside the
    adjoint of the current one) gives the sequential backward's bits."""
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.adjoint import Adjoint2D, probes_with_grad
    eps, sig, de, tau, m, ring = _case(72, 64, 6, 8)
    res = []
    for overlap in (False, True):
        s = BatchedFDTD2D(72, 64, 0.5e-3, 130, 6, ring[:3], ring, 2e9)
        s.set_dispersion(debye=[(de, tau)])
        adj = Adjoint2D(s, checkpoint_every=11, overlap=overlap)
        e = torch.tensor(eps, dtype=torch.float64, device="cuda", requires_grad=True)
        p = probes_with_grad(e, torch.tensor(sig, device="cuda"), adj, torch.tensor(de, device="cuda"),
                             torch.tensor(tau, device="cuda"))
        (p.double() ** 2).sum().backward()
        res.append(e.grad.clone())
    assert torch.equal(res[0], res[1])


def test_kept_segments_give_the_same_gradient(cuda_device):
    """Keeping 1, 2, 3 or all trailing segments (``keep_bytes``), with and
    without the two-stream backward, gives the same bits."""
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.adjoint import Adjoint2D, probes_with_grad
    eps, sig, de, tau, m, ring = _case(72, 64, 6, 8)
    res = []
    for keep in (0, 2, 3, 99):
        for overlap in (False, True):
            s = BatchedFDTD2D(72, 64, 0.5e-3, 130, 6, ring[:3], ring, 2e9)
            s.set_dispersion(debye=[(de, tau)])
            adj = Adjoint2D(s, checkpoint_every=11, overlap=overlap)
            s._build()
            adj.keep_bytes = keep * adj.segment_bytes()
            e = torch.tensor(eps, dtype=torch.float64, device="cuda", requires_grad=True)
            p = probes_with_grad(e, torch.tensor(sig, device="cuda"), adj, torch.tensor(de, device="cuda"),
                                 torch.tensor(tau, device="cuda"))
            assert len(adj._ckpt) == 12 - min(12, max(1, keep))      # 12 segments of 11 steps
            (p.double() ** 2).sum().backward()
            res.append(e.grad.clone())
    for r in res[1:]:
        assert torch.equal(res[0], r)


def test_adjoint_tile_height_setting(cuda_device):
    """``rows`` sets the adjoint launch's tile height; the gradient agrees
    with the automatic choice to FP32 rounding: the interior-tile path adds
    the adjoint curl terms in another order than the frame-tile path, so a
    cell that moves between the two kinds of tile rounds differently."""
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.adjoint import Adjoint2D, probes_with_grad
    eps, sig, de, tau, m, ring = _case(72, 64, 6, 8)
    res = []
    for rows in (0, 4, 12):
        s = BatchedFDTD2D(72, 64, 0.5e-3, 130, 6, ring[:3], ring, 2e9)
        s.set_dispersion(debye=[(de, tau)])
        adj = Adjoint2D(s, checkpoint_every=11, rows=rows)
        e = torch.tensor(eps, dtype=torch.float64, device="cuda", requires_grad=True)
        p = probes_with_grad(e, torch.tensor(sig, device="cuda"), adj, torch.tensor(de, device="cuda"),
                             torch.tensor(tau, device="cuda"))
        (p.double() ** 2).sum().backward()
        if rows:
            assert adj.launch_rows == rows
        res.append(e.grad.clone())
    scale = res[0].abs().max()
    for r in res[1:]:
        assert float((r - res[0]).abs().max() / scale) < 1e-5


@pytest.mark.parametrize("with_debye, K", [(True, 40), (False, 1)])
def test_lorentz_pole_gradient_matches_autograd(with_debye, K):
    """A Lorentz pole (with or without a Debye pole): the CUDA adjoint's
    gradients of sum(probes * G) with respect to eps_r, sigma, the Debye
    delta_eps and the Lorentz delta_eps against autograd through the FP64
    restatement (dispersive.py:278-299 recurrence, two time levels)."""
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.adjoint import Adjoint2D, probes_with_grad
    dev = torch.device("cuda")
    nx, ny, n, T, seed = 64, 60, 6, 150, 11   # sources outside the CPML strips
    eps, sig, de, tau, m, ring = _case(nx, ny, n, seed, True, 4)
    x, y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    ml = (x - nx // 2 - 2) ** 2 + (y - ny // 2 + 1) ** 2 <= 6 ** 2
    lde = np.where(ml, 3.0 + np.random.default_rng(seed).random((nx, ny)), 0.0)
    lw0, ldl = np.where(ml, 2 * np.pi * 5e9, 0.0), np.where(ml, 2 * np.pi * 0.6e9, 0.0)
    src, prb = ring[:3], ring
    f64 = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    G = torch.as_tensor(np.random.default_rng(seed + 100).standard_normal((3, len(prb), T)), device=dev)
    t = TorchFdtd2D(nx, ny, 0.5e-3, T, n, src, prb, 2e9, device=dev)
    e_, s_, l_ = (f64(a).requires_grad_(True) for a in (eps, sig, lde))
    d_ = f64(de).requires_grad_(True) if with_debye else None
    deb = [(d_, f64(tau))] if with_debye else []
    (t.run(e_, s_, deb, [(l_, f64(lw0), f64(ldl))]) * G).sum().backward()

    s = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, src, prb, 2e9)
    s.set_dispersion(debye=[(de, tau)] if with_debye else [], lorentz=[(lde, lw0, ldl)])
    adj = Adjoint2D(s, checkpoint_every=K)
    e2, s2, l2 = (f64(a).requires_grad_(True) for a in (eps, sig, lde))
    d2 = f64(de).requires_grad_(True) if with_debye else None
    p = probes_with_grad(e2, s2, adj, d2, f64(tau) if with_debye else None, lorentz_deps=(l2,))
    (p.double() * G).sum().backward()
    pairs = [("eps_r", e2.grad, e_.grad), ("sigma", s2.grad, s_.grad), ("lorentz_deps", l2.grad, l_.grad)]
    if with_debye:
        pairs.append(("deps", d2.grad, d_.grad))
    for name, got, want in pairs:
        err = rel_l2(got.cpu().numpy(), want.cpu().numpy())
        print(f"Lorentz adjoint (debye={with_debye}, K={K}) {name}: rel L2 {err:.2e}")
        assert err < TOL, (name, err)
