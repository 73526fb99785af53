"""The CUDA 3D adjoint against autograd through the PyTorch FP64 restatement
(itself pinned to the full 3D oracle and to central finite differences on
the CPU)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle.torch_fdtd3d import TorchFdtd3D

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _case(nx, ny, nz, seed, debye=True, nring=4):
    rng = np.random.default_rng(seed)
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    cx, cy, cz = nx // 2, ny // 2, nz // 2
    r = min(nx, ny, nz) // 5
    m = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 <= r ** 2
    eps = np.where(m, 6.0 + rng.random(m.shape), 1.0)
    sig = np.where(m, 0.3 + 0.2 * rng.random(m.shape), 0.0)
    de = np.where(m, 15.0 + 5 * rng.random(m.shape), 0.0) if debye else None
    tau = np.where(m, 8e-12, 0.0) if debye else None
    ang = 2 * np.pi * np.arange(nring) / nring
    ring = [(int(cx + (r + 4) * np.cos(a)), int(cy + (r + 4) * np.sin(a)), cz) for a in ang]
    return eps, sig, de, tau, m, ring


def _run_both(nx, ny, nz, n, T, seed, K, debye=True, ntx=3, nring=4):
    """Gradient of sum(probes * G) for a fixed random G through the CUDA
    adjoint and through autograd of the FP64 restatement."""
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.adjoint3d import Adjoint3D, probes_with_grad_3d
    dev = torch.device("cuda")
    eps, sig, de, tau, m, ring = _case(nx, ny, nz, seed, debye, nring)
    src, prb = ring[:ntx], ring
    f64 = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    G = torch.as_tensor(np.random.default_rng(seed + 100).standard_normal((ntx, len(prb), T)), device=dev)
    t = TorchFdtd3D(nx, ny, nz, 1e-3, T, n, src, prb, 2e9, device=dev)
    e_, s_ = f64(eps).requires_grad_(True), f64(sig).requires_grad_(True)
    d_ = f64(de).requires_grad_(True) if debye else None
    ref = (t.run(e_, s_, [(d_, f64(tau))] if debye else []) * G).sum()
    ref.backward()
    s = BatchedFDTD3D(nx, ny, nz, 1e-3, T, n, src, prb, 2e9)
    if debye:
        s.set_dispersion(debye=[(de, tau)])
    adj = Adjoint3D(s, checkpoint_every=K)
    e2, s2 = f64(eps).requires_grad_(True), f64(sig).requires_grad_(True)
    d2 = f64(de).requires_grad_(True) if debye else None
    val = (probes_with_grad_3d(e2, s2, adj, d2, f64(tau) if debye else None).double() * G).sum()
    val.backward()
    inner = np.zeros((nx, ny, nz), bool)
    inner[n + 1:nx - n, n + 1:ny - n, n + 1:nz - n] = True
    out = {"value": (float(val.detach()), float(ref.detach())), "eps_r": (e2.grad, e_.grad),
           "sigma": (s2.grad, s_.grad)}
    if debye:
        out["deps"] = (d2.grad, d_.grad)
    return out, inner


def _check(out, inner, keys, tol):
    v, vr = out["value"]
    assert abs(v - vr) <= 1e-4 * abs(vr) + 1e-30, (v, vr)
    for k in keys:
        g, gr = (x.detach().cpu().numpy() for x in out[k])
        assert np.all(g[~inner] == 0)
        err = rel_l2(g[inner], gr[inner])
        print(f"{k}: rel L2 vs autograd {err:.2e}")
        assert err < tol, (k, err)


def test_adjoint3d_vjp_matches_autograd(cuda_device):
    out, inner = _run_both(40, 36, 32, 4, 120, 1, K=25)
    _check(out, inner, ("eps_r", "sigma", "deps"), TOL)


def test_adjoint3d_one_segment(cuda_device):
    """checkpoint_every >= T: the forward's own saved segment serves the
    whole adjoint (no recompute)."""
    out, inner = _run_both(34, 34, 30, 3, 90, 2, K=500, ntx=4)
    _check(out, inner, ("eps_r", "sigma", "deps"), TOL)


def test_adjoint3d_two_tx_groups(cuda_device):
    """37 TX: two TX groups, whose per-group gradient sums are added."""
    out, inner = _run_both(36, 34, 30, 3, 60, 3, K=25, ntx=37, nring=37)
    _check(out, inner, ("eps_r", "sigma", "deps"), TOL)


def test_adjoint3d_without_dispersion(cuda_device):
    out, inner = _run_both(32, 30, 28, 3, 90, 4, K=20, debye=False)
    _check(out, inner, ("eps_r", "sigma"), TOL)


def test_adjoint3d_forward_equals_run(cuda_device):
    """The checkpointed forward gives the solver's own run() series bit for bit."""
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.adjoint3d import Adjoint3D
    eps, sig, de, tau, m, ring = _case(30, 28, 26, 5)
    mk = lambda: BatchedFDTD3D(30, 28, 26, 1e-3, 70, 3, ring[:2], ring, 2e9)
    a = mk()
    a._eps_r[:], a._sigma_e[:] = eps, sig
    a.set_dispersion(debye=[(de, tau)])
    a.run()
    b = mk()
    b.set_dispersion(debye=[(de, tau)])
    adj = Adjoint3D(b, checkpoint_every=16)
    adj.set_parameters(eps, sig, de, tau)
    p = adj.forward()
    assert torch.equal(p, a.probe_data[:, :len(ring)])


def test_adjoint3d_checkpoint_interval_does_not_change_the_gradient(cuda_device):
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.adjoint3d import Adjoint3D, probes_with_grad_3d
    eps, sig, de, tau, m, ring = _case(30, 28, 26, 6)
    res = []
    for K in (7, 40, 100):
        s = BatchedFDTD3D(30, 28, 26, 1e-3, 80, 3, ring[:3], ring, 2e9)
        s.set_dispersion(debye=[(de, tau)])
        adj = Adjoint3D(s, checkpoint_every=K)
        e = torch.tensor(eps, dtype=torch.float64, device="cuda", requires_grad=True)
        p = probes_with_grad_3d(e, torch.tensor(sig, device="cuda"), adj, torch.tensor(de, device="cuda"),
                                torch.tensor(tau, device="cuda"))
        (p.double() ** 2).sum().backward()
        res.append(e.grad.clone())
    assert torch.equal(res[0], res[1]) and torch.equal(res[0], res[2])


def test_interior_only_save_pass_is_bit_identical(cuda_device):
    """The recompute mode (CPML shell skipped) stores the same E slots and
    leaves the same E, H box, currents and probes as a full save pass."""
    import ctypes as C
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200._lib import check, lib
    from ceep_b200.adjoint3d import interior_e, save_slot_shape
    eps, sig, de, tau, m, ring = _case(30, 28, 26, 9)
    out = []
    for interior_only in (0, 1):
        s = BatchedFDTD3D(30, 28, 26, 1e-3, 60, 3, ring[:3], ring, 2e9)
        s._eps_r[:], s._sigma_e[:] = eps, sig
        s.set_dispersion(debye=[(de, tau)])
        s.advance(0, 20)
        seg = torch.zeros((41,) + save_slot_shape(s), dtype=torch.float32, device="cuda")
        st = torch.cuda.current_stream()
        check(lib().ceep3d_plan_run_save(s._plan, 20, 40, C.c_void_p(st.cuda_stream), 1, seg.data_ptr(), 20,
                                         interior_only), "ceep3d_plan_run_save")
        torch.cuda.synchronize()
        out.append((seg, {k: v.clone() for k, v in s._f.items()}, s._j.clone(), s.probe_data.clone()))
    (sa, fa, ja, pa), (sb, fb, jb, pb) = out
    n = 3
    box = (slice(None), slice(n, 26 - n), slice(n, 28 - n), slice(n, 30 - n))
    assert torch.equal(sa, sb) and torch.equal(ja, jb) and torch.equal(pa, pb)
    for k in ("ex", "ey", "ez"):
        assert torch.equal(fa[k], fb[k])
    for k in ("hx", "hy", "hz"):
        assert torch.equal(fa[k][box], fb[k][box])
    # the last slot is the interior E of the last step before its source: it
    # differs from the final state at the three source cells only
    for c, k in enumerate(("ex", "ey", "ez")):
        d = (sa[40, c] != interior_e(s, fa[k])).sum().item()
        assert d <= (3 if k == "ez" else 0), (k, d)


def test_adjoint3d_overlapped_recompute_gives_the_same_gradient(cuda_device):
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.adjoint3d import Adjoint3D, probes_with_grad_3d
    eps, sig, de, tau, m, ring = _case(30, 28, 26, 10)
    res = []
    for overlap in (False, True):
        s = BatchedFDTD3D(30, 28, 26, 1e-3, 75, 3, ring[:3], ring, 2e9)
        s.set_dispersion(debye=[(de, tau)])
        adj = Adjoint3D(s, checkpoint_every=9, overlap=overlap)
        e = torch.tensor(eps, dtype=torch.float64, device="cuda", requires_grad=True)
        p = probes_with_grad_3d(e, torch.tensor(sig, device="cuda"), adj, torch.tensor(de, device="cuda"),
                                torch.tensor(tau, device="cuda"))
        (p.double() ** 2).sum().backward()
        res.append(e.grad.clone())
    assert torch.equal(res[0], res[1])


def test_adjoint3d_kept_segments_give_the_same_gradient(cuda_device):
    """Keeping 1, 3 or all trailing segments (``keep_bytes``), with and
    without the two-stream backward, gives the same bits."""
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.adjoint3d import Adjoint3D, probes_with_grad_3d
    eps, sig, de, tau, m, ring = _case(30, 28, 26, 10)
    res = []
    for keep in (0, 3, 99):
        for overlap in (False, True):
            s = BatchedFDTD3D(30, 28, 26, 1e-3, 75, 3, ring[:3], ring, 2e9)
            s.set_dispersion(debye=[(de, tau)])
            s._build()
            adj = Adjoint3D(s, checkpoint_every=9, overlap=overlap)
            adj.keep_bytes = keep * adj.segment_bytes()
            e = torch.tensor(eps, dtype=torch.float64, device="cuda", requires_grad=True)
            p = probes_with_grad_3d(e, torch.tensor(sig, device="cuda"), adj, torch.tensor(de, device="cuda"),
                                    torch.tensor(tau, device="cuda"))
            assert len(adj._ckpt) == 9 - min(9, max(1, keep))     # 9 segments of 9 steps (the last 3)
            (p.double() ** 2).sum().backward()
            res.append(e.grad.clone())
    for r in res[1:]:
        assert torch.equal(res[0], r)
