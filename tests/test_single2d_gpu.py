"""The non-batched FDTD2D on the GPU against the reference's own run
(tests/golden/single2d.npz: TMz / TEz, CFS-CPML, PEC, Mur, every source
component) and against the oracle, at the 1e-4 relative L2 bar."""
import os
import sys

import numpy as np
import pytest
import torch

from conftest import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import SINGLE2D  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = 1e-4
GOLD = np.load(os.path.join(HERE, "golden", "single2d.npz"))
FIELDS = {"TMZ": ("ez", "hx", "hy"), "TEZ": ("hz", "ex", "ey")}


def build(case, **kw):
    from ceep_b200 import fdtd2d as F
    name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats = case
    cfg = F.SimulationConfig(grid=F.GridConfig(nx=nx, ny=ny, dx=1e-3, dy=0.8e-3),
                             mode=getattr(F.SimulationMode, mode), total_steps=steps)
    boundaries = []
    for b in bcs:
        if b[0] == "cpml":
            boundaries.append(F.CPML(thickness=b[1], order=b[2], sigma_factor=b[3], alpha_max=b[4], kappa_max=b[5]))
        else:
            boundaries.append(F.MurABC() if b[0] == "mur" else F.PEC())
    sources = []
    for sp in srcs:
        if sp[0] == "gauss":
            sources.append(F.GaussianSource(x=sp[1], y=sp[2], frequency_max=sp[3], amplitude=sp[4],
                                            delay_factor=sp[5], field_component=sp[6]))
        elif sp[0] == "modgauss":
            sources.append(F.ModulatedGaussianSource(x=sp[1], y=sp[2], frequency=sp[3], bandwidth=sp[4],
                                                     amplitude=sp[5], delay_factor=sp[6], field_component=sp[7]))
        else:
            sources.append(F.SinusoidalSource(x=sp[1], y=sp[2], frequency=sp[3], amplitude=sp[4],
                                              field_component=sp[5]))
    s = F.FDTD2D(cfg, sources=sources, boundaries=boundaries, record_field=rec, record_interval=interval,
                 probe_points=[tuple(p) for p in prbs], **kw)
    for m in mats:
        if m[0] == "circle":
            s.grid.set_material_circle(m[1], m[2], m[3], eps_r=m[4], mu_r=m[5], sigma_e=m[6], sigma_m=m[7])
        else:
            s.grid.set_material_region(m[1], m[2], m[3], m[4], eps_r=m[5], mu_r=m[6], sigma_e=m[7], sigma_m=m[8])
    return s


@pytest.mark.parametrize("case", SINGLE2D, ids=[c[0] for c in SINGLE2D])
def test_fdtd2d_matches_reference(cuda_device, case):
    name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats = case
    s = build(case)
    s.run()
    assert s.current_step == steps
    got = np.array([s.probe_data[tuple(p)] for p in prbs])
    ref = GOLD[f"{name}_probes"]
    err = rel_l2(got, ref)
    print(f"{name}: probes rel L2 {err:.2e}")
    assert err < TOL
    for f in FIELDS[mode]:
        e = rel_l2(getattr(s.grid, f).double().cpu().numpy(), GOLD[f"{name}_{f}"])
        assert e < TOL, (f, e)
    snaps = GOLD[f"{name}_snapshots"]
    assert len(s.field_snapshots) == len(snaps)
    if len(snaps):
        assert rel_l2(np.array(s.field_snapshots), snaps) < TOL


def test_step_by_step_equals_run_and_graph_equals_stream(cuda_device):
    case = SINGLE2D[1]
    a = build(case)
    a.run()
    first = {f: getattr(a.grid, f).clone() for f in FIELDS[case[1]]}
    a.reset()
    a.run()                # the same range again: captured and replayed as a graph
    for f in FIELDS[case[1]]:
        assert torch.equal(first[f], getattr(a.grid, f))
    b = build(case, use_graph=False)
    for _ in range(case[4]):
        b.step()
    c = build(case)
    c.run(100)
    c.run(case[4] - 100)   # grows past nothing, second graph
    for other in (b, c):
        for f in FIELDS[case[1]]:
            assert torch.equal(getattr(a.grid, f), getattr(other.grid, f))
        assert a.probe_data == other.probe_data
        assert all(np.array_equal(x, y) for x, y in zip(a.field_snapshots, other.field_snapshots))


def test_run_past_the_configured_steps(cuda_device):
    """Running more steps than config.num_steps regrows the waveform and
    record buffers and keeps what was recorded."""
    case = SINGLE2D[2]
    a = build(case)
    a.run(case[4] + 60)
    b = build(case)
    b.run()
    b.run(60)
    assert a.probe_data == b.probe_data
    assert torch.equal(a.grid.ez, b.grid.ez)


def test_dft_monitor_matches_oracle_series(cuda_device):
    from ceep_b200 import fdtd2d as F
    from oracle.fdtd2d_single import Single2DOracle
    case = SINGLE2D[0]
    name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats = case
    freqs = np.array([3e9, 6e9, 9e9])
    mon = F.DFTMonitor(freqs, (slice(20, 26), slice(30, 33)), component="Ez")
    pt = F.DFTMonitor(freqs, (40, 12), component="Ez")
    s = build(case)
    s.dft_monitors = [mon, pt]
    s.initialize(s.config)
    for m in mats:
        if m[0] == "circle":
            s.grid.set_material_circle(m[1], m[2], m[3], eps_r=m[4], mu_r=m[5], sigma_e=m[6], sigma_m=m[7])
        else:
            s.grid.set_material_region(m[1], m[2], m[3], m[4], eps_r=m[5], mu_r=m[6], sigma_e=m[7], sigma_m=m[8])
    s.run()
    cells = [(i, j) for i in range(20, 26) for j in range(30, 33)] + [(40, 12)]
    w = GOLD[f"{name}_waveforms"]
    g = lambda k: GOLD[f"{name}_{k}"]
    o = Single2DOracle(nx, ny, 1e-3, 0.8e-3, float(g("dt")), mode, g("ca"), g("cb"), g("da"), g("db"),
                       [(sp[1], sp[2], sp[-1], w[k]) for k, sp in enumerate(srcs)], bcs, cells, "Ez", 10 ** 9)
    o.run(steps)
    ser = np.array([o.probe_data[c] for c in cells])                      # (cells, T)
    t = np.arange(steps) * float(g("dt"))
    ph = 2 * np.pi * freqs[:, None] * t[None, :]
    ref = (np.cos(ph) - 1j * np.sin(ph)) @ ser.T * float(g("dt"))         # (F, cells)
    got = np.concatenate([mon.get_complex_field().reshape(3, -1), pt.get_complex_field().reshape(3, 1)], 1)
    assert rel_l2(np.concatenate([got.real, got.imag]), np.concatenate([ref.real, ref.imag])) < TOL


# Grids large enough for an interior rectangle of walk blocks (the golden
# cases above are small enough that every block is a frame block): an even
# ny runs the two-column interior walk (TMz and TEz), an odd ny the
# one-column one.  Sources sit on even and odd columns, on a pair's first and
# last owned columns (74 and 135: the rectangle starts at column 12 for
# CPML 10) and in the frame; probes sit beside the rectangle and on a pair
# boundary.
INTERIOR = [
    ("tmz_pairs", "TMZ", 300, 262, 130, [("cpml", 10, 3, 1.0, 0.05, 1.0)],
     [("gauss", 150, 100, 20e9, 1.0, 6.0, "Ez"), ("gauss", 200, 131, 15e9, 0.8, 5.0, "Ez"),
      ("gauss", 140, 74, 20e9, 0.5, 6.0, "Ez"), ("gauss", 180, 135, 20e9, 0.5, 6.0, "Ez"),
      ("gauss", 20, 30, 20e9, 1.0, 6.0, "Ez")],
     [(150, 100), (170, 140), (129, 11), (129, 73), (255, 200), (12, 250), (289, 130)], "Ez", 40,
     [("circle", 150, 131, 40, 4.0, 1.0, 0.2, 0.0), ("region", 130, 170, 60, 70, 2.5, 1.0, 0.05, 0.0)]),
    ("tmz_odd_ny", "TMZ", 290, 259, 120, [("cpml", 10, 3, 1.0, 0.05, 1.0)],
     [("gauss", 150, 100, 20e9, 1.0, 6.0, "Ez"), ("gauss", 190, 133, 20e9, 1.0, 6.0, "Ez")],
     [(150, 100), (170, 140), (250, 251)], "Ez", 60,
     [("circle", 145, 129, 35, 4.0, 1.0, 0.2, 0.0)]),
    ("tez_interior", "TEZ", 280, 250, 120, [("cpml", 10, 3, 1.0, 0.05, 1.0)],
     [("gauss", 150, 100, 20e9, 1.0, 6.0, "Hz"), ("gauss", 180, 131, 15e9, 0.7, 5.0, "Ex"),
      ("sin", 140, 90, 12e9, 0.3, "Ey")],
     [(150, 100), (170, 140), (20, 20)], "Hz", 40,
     [("circle", 140, 125, 35, 5.0, 1.0, 0.3, 0.0)]),
    ("tez_odd_ny", "TEZ", 270, 251, 100, [("cpml", 10, 3, 1.0, 0.05, 1.0)],
     [("gauss", 140, 101, 20e9, 1.0, 6.0, "Hz"), ("gauss", 170, 130, 15e9, 0.7, 5.0, "Ey")],
     [(140, 101), (160, 140), (260, 240)], "Ex", 50,
     [("circle", 135, 125, 30, 5.0, 1.0, 0.3, 0.0)]),
]


@pytest.mark.parametrize("case", INTERIOR, ids=[c[0] for c in INTERIOR])
def test_interior_walks_match_oracle(cuda_device, case):
    from oracle.fdtd2d_single import Single2DOracle
    name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats = case
    s = build(case)
    s.run()
    g, dt = s.grid, s.config.dt
    waves = [np.array([src.value_at(k, dt) for k in range(steps)]) for src in s.sources]
    o = Single2DOracle(nx, ny, 1e-3, 0.8e-3, dt, mode, g._ca, g._cb, g._da, g._db,
                       [(sp[1], sp[2], sp[-1], waves[k]) for k, sp in enumerate(srcs)], bcs, prbs, rec, interval)
    o.run(steps)
    got = np.array([s.probe_data[tuple(p)] for p in prbs])
    ref = np.array([o.probe_data[tuple(p)] for p in prbs])
    assert rel_l2(got, ref) < TOL, rel_l2(got, ref)
    names = {"ez": "Ez", "hx": "Hx", "hy": "Hy", "hz": "Hz", "ex": "Ex", "ey": "Ey"}
    for f in FIELDS[mode]:
        e = rel_l2(getattr(s.grid, f).double().cpu().numpy(), o.f[names[f]])
        assert e < TOL, (f, e)
    assert len(s.field_snapshots) == len(o.snapshots)
    assert rel_l2(np.array(s.field_snapshots), np.array(o.snapshots)) < TOL
