"""Parity of the CUDA 2D path with the reference (golden fixtures) and the oracle.

Tolerance: the north-star bar is 1e-4 relative L2 against the reference's
FP32 run; every test below also asserts the error against the FP64 result.
"""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle.fdtd2d import Fdtd2DOracle

pytestmark = pytest.mark.gpu
TOL = 1e-4

SMALL = dict(nx=48, ny=40, dx=0.5e-3, total_steps=260, cpml_thickness=6, frequency=2e9)
SMALL_SRC = [(20, 18), (8, 30), (40, 6)]
SMALL_PRB = [(20, 18), (7, 7), (41, 33), (24, 2)]


def _solver(**kw):
    from ceep_b200 import BatchedFDTD2D
    return BatchedFDTD2D(**kw)


def _probes(out, B, P):
    return np.array([[out[b][p] for p in range(P)] for b in range(B)])


def test_small_against_reference_fp32_and_fp64(cuda_device):
    g64, g32 = load_golden("fdtd2d_small_float64"), load_golden("fdtd2d_small_float32")
    s = _solver(source_positions=SMALL_SRC, probe_positions=SMALL_PRB, **SMALL)
    s._eps_r[:] = g64["eps_r"]
    s._sigma_e[:] = g64["sigma_e"]
    out = _probes(s.run(), 3, 4)
    assert rel_l2(out, g32["probes"]) < TOL
    assert rel_l2(out, g64["probes"]) < TOL
    # the full state, psi included, in the reference layout
    assert rel_l2(s.ez.cpu().numpy(), g64["ez"]) < TOL
    assert rel_l2(s.hx.cpu().numpy(), g64["hx"]) < TOL
    assert rel_l2(s.hy.cpu().numpy(), g64["hy"]) < TOL
    cur = s._cur()
    n, nx, ny = 6, 48, 40
    psi_hy = s._psi_hy[cur][0, :, :, :3].permute(2, 1, 0).cpu().numpy()   # (B, 2n, ny)
    assert rel_l2(psi_hy[:, :n], g64["psi_hxy_lo"]) < TOL
    assert rel_l2(psi_hy[:, n:2 * n - 1], g64["psi_hxy_hi"][:, :n - 1]) < TOL
    psi_ezy = s._psi_ezy[cur][0, :, :, :3].permute(2, 1, 0).cpu().numpy()   # (B, nx, 2n)
    assert rel_l2(psi_ezy[:, :, :n], g64["psi_ezy_lo"]) < TOL
    assert rel_l2(psi_ezy[:, :, n:], g64["psi_ezy_hi"]) < TOL


def test_cfg1_against_reference(cuda_device):
    g64, g32 = load_golden("fdtd2d_cfg1_float64"), load_golden("fdtd2d_cfg1_float32")
    pos = [tuple(int(v) for v in p) for p in g64["positions"]]
    s = _solver(nx=200, ny=200, dx=0.5e-3, total_steps=400, cpml_thickness=15, source_positions=pos,
                probe_positions=pos, frequency=2e9)
    s.set_material_circle(100, 100, 40, 40.0, 0.5)
    out = _probes(s.run(), 8, 8)
    e32, e64 = rel_l2(out, g32["probes"]), rel_l2(out, g64["probes"])
    print(f"cfg1: rel L2 vs reference FP32 {e32:.3e}, vs FP64 {e64:.3e}")
    assert e32 < TOL and e64 < TOL


@pytest.mark.parametrize("kind", ["brain", "hemorrhage"])
def test_ceep_results_json(cuda_device, kind):
    g = load_golden("ceep_results")
    nx = 64
    s = _solver(nx=nx, ny=nx, dx=0.5e-3, total_steps=100, cpml_thickness=10, source_positions=[(32, 32)],
                probe_positions=[(32, 32)], frequency=2e9)
    x, y = np.ogrid[:nx, :nx]
    m = np.sqrt((x - 32) ** 2 + (y - 32) ** 2) < 20
    s._eps_r[m], s._sigma_e[m] = 50.0, 1.5
    if kind == "hemorrhage":
        m = np.sqrt((x - 40) ** 2 + (y - 37) ** 2) < 10
        s._eps_r[m], s._sigma_e[m] = 60.0, 2.0
    out = s.run()[0][0]
    assert rel_l2(out, g[kind]) < TOL


def test_run_cpu_variant(cuda_device):
    g = load_golden("fdtd2d_runcpu")
    s = _solver(nx=40, ny=36, dx=0.5e-3, total_steps=150, cpml_thickness=5,
                source_positions=[(10, 12), (30, 20), (19, 30)], probe_positions=[(10, 12), (25, 25), (5, 31)],
                frequency=2e9)
    s._eps_r[:], s._sigma_e[:] = g["eps_r"], g["sigma_e"]
    assert rel_l2(_probes(s.run_cpu(), 3, 3), g["probes"]) < TOL


CASES = [
    # nx, ny, n, steps, B, seed
    (37, 29, 3, 120, 1, 0),
    (50, 44, 5, 200, 3, 1),
    (64, 40, 0, 90, 5, 2),
    (33, 61, 2, 150, 8, 3),
    (70, 70, 8, 160, 13, 4),
    (41, 47, 6, 140, 16, 5),
    (45, 39, 4, 100, 20, 6),
    (30, 34, 3, 80, 33, 7),
]


def _random_case(nx, ny, n, steps, B, seed, pml_sources=False):
    """Sources inside the interior region (the reference's strip update is
    unstable for long runs with a source inside the CPML); probes anywhere,
    edges and strips included."""
    rng = np.random.default_rng(seed)
    lo = 0 if pml_sources else n + 1
    src = [(int(rng.integers(lo, nx - lo)), int(rng.integers(lo, ny - lo))) for _ in range(B)]
    if pml_sources and B > 1:
        src[0] = (0, ny - 1)
        src[1] = (1, n // 2)
    prb = [(int(rng.integers(0, nx)), int(rng.integers(0, ny))) for _ in range(4)] + [src[-1], (nx - 1, 1)]
    eps = 1.0 + 30.0 * (rng.random((nx, ny)) < 0.3) * rng.random((nx, ny))
    sig = 0.8 * rng.random((nx, ny)) * (eps > 1)
    return src, prb, eps, sig


@pytest.mark.parametrize("case", CASES)
def test_random_against_oracle(cuda_device, case):
    nx, ny, n, steps, B, seed = case
    src, prb, eps, sig = _random_case(*case)
    o = Fdtd2DOracle(nx, ny, 0.5e-3, steps, n, src, prb, 2e9, eps_r=eps, sigma_e=sig)
    o.run()
    s = _solver(nx=nx, ny=ny, dx=0.5e-3, total_steps=steps, cpml_thickness=n, source_positions=src,
                probe_positions=prb, frequency=2e9)
    s._eps_r[:], s._sigma_e[:] = eps, sig
    out = _probes(s.run(), B, len(prb))
    assert rel_l2(out, o.probe_data) < TOL
    assert rel_l2(s.ez.cpu().numpy(), o.ez) < TOL
    assert rel_l2(s.hx.cpu().numpy(), o.hx) < TOL
    assert rel_l2(s.hy.cpu().numpy(), o.hy) < TOL


@pytest.mark.parametrize("case", [(40, 36, 4, 40, 5, 31), (52, 48, 6, 30, 9, 32), (30, 30, 0, 60, 3, 33)])
def test_sources_in_cpml_and_on_edges_short_runs(cuda_device, case):
    nx, ny, n, steps, B, seed = case
    src, prb, eps, sig = _random_case(*case, pml_sources=True)
    o = Fdtd2DOracle(nx, ny, 0.5e-3, steps, n, src, prb, 2e9, eps_r=eps, sigma_e=sig)
    o.run()
    assert np.isfinite(o.ez).all() and np.abs(o.ez).max() < 1e20
    s = _solver(nx=nx, ny=ny, dx=0.5e-3, total_steps=steps, cpml_thickness=n, source_positions=src,
                probe_positions=prb, frequency=2e9)
    s._eps_r[:], s._sigma_e[:] = eps, sig
    out = _probes(s.run(), B, len(prb))
    assert rel_l2(out, o.probe_data) < TOL
    assert rel_l2(s.ez.cpu().numpy(), o.ez) < TOL


@pytest.mark.parametrize("rows", [1, 3, 16, 64])
def test_partition_independent_bitwise(cuda_device, rows):
    src, prb, eps, sig = _random_case(57, 49, 5, 90, 6, 11)
    ref = None
    for r in (rows, 7):
        s = _solver(nx=57, ny=49, dx=0.5e-3, total_steps=90, cpml_thickness=5, source_positions=src,
                    probe_positions=prb, frequency=2e9, rows_per_block=r)
        s._eps_r[:], s._sigma_e[:] = eps, sig
        s.run()
        cur = (s.probe_data.clone(), s.ez.clone())
        if ref is None:
            ref = cur
        else:
            assert torch.equal(ref[0], cur[0]) and torch.equal(ref[1], cur[1])


def test_graph_equals_stream_launches(cuda_device):
    src, prb, eps, sig = _random_case(60, 52, 6, 101, 9, 12)
    res = []
    for g in (True, False):
        s = _solver(nx=60, ny=52, dx=0.5e-3, total_steps=101, cpml_thickness=6, source_positions=src,
                    probe_positions=prb, frequency=2e9, use_graph=g)
        s._eps_r[:], s._sigma_e[:] = eps, sig
        s.run()
        res.append(s.probe_data.clone())
    assert torch.equal(res[0], res[1])


def test_tx_permutation_and_subset_bitwise(cuda_device):
    """Each transmit event is computed independently with the same arithmetic,
    so permuting or splitting the batch changes nothing, bit for bit."""
    src, prb, eps, sig = _random_case(66, 58, 7, 120, 12, 13)
    kw = dict(nx=66, ny=58, dx=0.5e-3, total_steps=120, cpml_thickness=7, probe_positions=prb, frequency=2e9)
    full = _solver(source_positions=src, **kw)
    full._eps_r[:], full._sigma_e[:] = eps, sig
    full.run()
    perm = np.random.default_rng(1).permutation(12)
    ps = _solver(source_positions=[src[i] for i in perm], **kw)
    ps._eps_r[:], ps._sigma_e[:] = eps, sig
    ps.run()
    assert torch.equal(full.probe_data[perm], ps.probe_data)
    sub = _solver(source_positions=src[3:5], **kw)
    sub._eps_r[:], sub._sigma_e[:] = eps, sig
    sub.run()
    assert torch.equal(full.probe_data[3:5], sub.probe_data)


def test_second_run_continues_like_reference(cuda_device):
    """A second run() keeps the fields and restarts the waveform/probe index
    (fdtd_2d_batched.py:419-420), for odd and even step counts."""
    for steps in (51, 60):
        src, prb, eps, sig = _random_case(44, 40, 4, steps, 3, 14)
        o = Fdtd2DOracle(44, 40, 0.5e-3, steps, 4, src, prb, 2e9, eps_r=eps, sigma_e=sig)
        o.run()
        o.step_index = 0
        o.run()
        s = _solver(nx=44, ny=40, dx=0.5e-3, total_steps=steps, cpml_thickness=4, source_positions=src,
                    probe_positions=prb, frequency=2e9)
        s._eps_r[:], s._sigma_e[:] = eps, sig
        s.run()
        out = _probes(s.run(), 3, len(prb))
        assert rel_l2(out, o.probe_data) < TOL


def test_linearity_at_full_size(cuda_device):
    """Size-independent property at the 600x600x16 head-imaging size: the
    response is linear in the source waveform."""
    from ceep_b200 import physics
    nx = 600
    ang = 2 * np.pi * np.arange(16) / 16
    pos = [(int(300 + 200 * np.cos(a)), int(300 + 200 * np.sin(a))) for a in ang]
    steps = 200
    s1 = _solver(nx=nx, ny=nx, dx=0.5e-3, total_steps=steps, cpml_thickness=15, source_positions=pos,
                 probe_positions=pos, frequency=2e9)
    s1.set_material_circle(300, 300, 150, 40.0, 0.5)
    w = physics.gaussian_derivative(steps, s1.dt, 2e9) * 1e-9 + 1.0 * np.sin(np.arange(steps) * 0.3)
    a = _solver(nx=nx, ny=nx, dx=0.5e-3, total_steps=steps, cpml_thickness=15, source_positions=pos,
                probe_positions=pos, frequency=2e9, waveform=w)
    b = _solver(nx=nx, ny=nx, dx=0.5e-3, total_steps=steps, cpml_thickness=15, source_positions=pos,
                probe_positions=pos, frequency=2e9, waveform=4.0 * w)
    for s in (a, b):
        s.set_material_circle(300, 300, 150, 40.0, 0.5)
        s.run()
    # scaling by a power of two commutes with every rounding except where a
    # product underflows into the subnormal range (the far tail of the wave
    # front); those last-bit differences then travel with the wave, so the
    # check is a tight relative bound rather than bit equality
    pa, pb = 4.0 * a.probe_data, b.probe_data
    assert rel_l2(pa.cpu().numpy(), pb.cpu().numpy()) < 1e-6
    assert torch.isfinite(a.probe_data).all()


def test_ade_against_reference_composition(cuda_device):
    g = load_golden("ade2d_small")
    lor = g["lor_mask"]
    deb = g["deb_mask"] & ~lor
    s = _solver(nx=44, ny=40, dx=0.5e-3, total_steps=220, cpml_thickness=5, source_positions=[(14, 20), (30, 12)],
                probe_positions=[(14, 20), (30, 12), (22, 30)], frequency=2e9)
    s._eps_r[:], s._sigma_e[:] = g["eps_r"], g["sigma_e"]
    s.set_dispersion(debye=[(np.where(deb, 30.0, 0.0), np.where(deb, 9e-12, 0.0))],
                     lorentz=[(np.where(lor, 5.0, 0.0), np.where(lor, 2 * np.pi * 6e9, 0.0),
                               np.where(lor, 2 * np.pi * 0.5e9, 0.0))])
    out = _probes(s.run(), 2, 3)
    assert rel_l2(out, g["probes"]) < TOL


@pytest.mark.parametrize("kinds", [("d", "d"), ("l", "l"), ("d",), ("l",)])
def test_ade_pole_mixes_against_oracle(cuda_device, kinds):
    nx, ny, n, T, B = 52, 46, 5, 180, 5
    rng = np.random.default_rng(21)
    x, y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    m = (x - 26) ** 2 + (y - 23) ** 2 <= 12 ** 2
    deb, lor = [], []
    for k in kinds:
        if k == "d":
            deb.append((np.where(m, rng.uniform(10, 45), 0.0), np.where(m, rng.uniform(5e-12, 15e-12), 0.0)))
        else:
            lor.append((np.where(m, rng.uniform(1, 8), 0.0), np.where(m, 2 * np.pi * rng.uniform(1e9, 20e9), 0.0),
                        np.where(m, 2 * np.pi * rng.uniform(0.1e9, 1e9), 0.0)))
    eps = np.where(m, 6.0, 1.0)
    sig = np.where(m, 0.7, 0.0)
    src = [(int(rng.integers(8, 44)), int(rng.integers(8, 38))) for _ in range(B)]
    prb = src[:3] + [(26, 23)]
    o = Fdtd2DOracle(nx, ny, 0.5e-3, T, n, src, prb, 2e9, eps_r=eps, sigma_e=sig,
                     dispersion={"debye": deb, "lorentz": lor})
    o.run()
    s = _solver(nx=nx, ny=ny, dx=0.5e-3, total_steps=T, cpml_thickness=n, source_positions=src,
                probe_positions=prb, frequency=2e9)
    s._eps_r[:], s._sigma_e[:] = eps, sig
    s.set_dispersion(debye=deb, lorentz=lor)
    out = _probes(s.run(), B, len(prb))
    assert rel_l2(out, o.probe_data) < TOL


def test_autotuned_tile_height_gives_the_same_bits():
    """BatchedFDTD2D.autotune times each candidate tile height and keeps the
    fastest; the probe series and fields equal a run at the automatic height."""
    from ceep_b200 import BatchedFDTD2D
    nx, ny, T = 120, 104, 90
    src = [(30, 30), (90, 70), (60, 52), (40, 80), (85, 25)]
    def mk():
        s = BatchedFDTD2D(nx, ny, 0.5e-3, T, 10, src, src, 2e9)
        x, y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
        m = (x - 60) ** 2 + (y - 52) ** 2 <= 20 ** 2
        s._eps_r[m], s._sigma_e[m] = 12.0, 0.4
        return s
    a = mk()
    a.run()
    b = mk()
    t = b.autotune(candidates=(6, 9, 14), steps=20)
    assert set(t) == {6, 9, 14} and b.rows_per_block in t
    b.run()
    assert torch.equal(a.probe_data, b.probe_data) and torch.equal(a.ez, b.ez)


@pytest.mark.parametrize("poles, rows", [("debye", 0), ("lorentz", 6), ("none", 9)])
def test_frame_split_gives_the_same_bits(poles, rows):
    """Two steps per launch as a frame-tile kernel beside an interior-tile
    kernel (the default) and as one kernel give the same probe series,
    fields and currents, with and without ADE poles and for several tile
    heights (an odd step count ends on a one-step launch)."""
    from ceep_b200 import BatchedFDTD2D
    nx, ny, T = 200, 176, 61
    src = [(40, 40), (160, 130), (100, 88), (60, 140), (150, 30)]
    x, y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    m = (x - 100) ** 2 + (y - 88) ** 2 <= 40 ** 2
    runs = []
    for split in (True, False):
        s = BatchedFDTD2D(nx, ny, 0.5e-3, T, 12, src, src, 2e9, rows_per_block=rows)
        s._eps_r[m], s._sigma_e[m] = 12.0, 0.4
        if poles == "debye":
            s.set_dispersion(debye=[(np.where(m, 20.0, 0.0), np.where(m, 8e-12, 0.0))])
        elif poles == "lorentz":
            s.set_dispersion(lorentz=[(np.where(m, 3.0, 0.0), np.where(m, 2 * np.pi * 3e9, 0.0),
                                       np.where(m, 1e9, 0.0))])
        s.set_frame_split(split)
        s.run()
        runs.append(s)
    a, b = runs
    assert torch.equal(a.probe_data, b.probe_data) and torch.equal(a.ez, b.ez)
    assert torch.equal(a.hx, b.hx) and torch.equal(a.hy, b.hy)
    # kernel launches: two per two-step launch when split, plus the last single step
    assert a.launches(T) == 2 * (T // 2) + T % 2 and b.launches(T) == T // 2 + T % 2
