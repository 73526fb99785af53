"""The non-batched 2D oracle (TMz / TEz, CFS-CPML, PEC, Mur) against the
reference's own FDTD2D run (tests/golden/single2d.npz), and host-side checks
of the drop-in API that need no GPU."""
import os
import sys

import numpy as np
import torch
import pytest

from oracle.fdtd2d_single import Single2DOracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import SINGLE2D  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "single2d.npz"))
FIELDS = {"TMZ": ("ez", "hx", "hy"), "TEZ": ("hz", "ex", "ey")}
NAMES = {"ez": "Ez", "hx": "Hx", "hy": "Hy", "hz": "Hz", "ex": "Ex", "ey": "Ey"}


def _comp(sp):
    return sp[-1]


def run_oracle(case):
    name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats = case
    g = lambda k: GOLD[f"{name}_{k}"]
    w = g("waveforms")
    sources = [(sp[1], sp[2], _comp(sp), w[k]) for k, sp in enumerate(srcs)]
    o = Single2DOracle(nx, ny, 1e-3, 0.8e-3, float(g("dt")), mode, g("ca"), g("cb"), g("da"), g("db"),
                       sources, bcs, [tuple(p) for p in prbs], rec, interval)
    o.run(steps)
    return o


@pytest.mark.parametrize("case", SINGLE2D, ids=[c[0] for c in SINGLE2D])
def test_oracle_matches_reference_fdtd2d(case):
    name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats = case
    o = run_oracle(case)
    ref = GOLD[f"{name}_probes"]
    got = np.array([o.probe_data[tuple(p)] for p in prbs])
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(got - ref).max() <= 1e-12 * scale
    for f in FIELDS[mode]:
        r = GOLD[f"{name}_{f}"]
        assert np.abs(o.f[NAMES[f]] - r).max() <= 1e-12 * max(np.abs(r).max(), 1e-300)
    snaps = GOLD[f"{name}_snapshots"]
    assert len(o.snapshots) == len(snaps)
    if len(snaps):
        assert np.abs(np.array(o.snapshots) - snaps).max() <= 1e-12 * np.abs(snaps).max()


def test_desc_layout_matches_the_library():
    from ceep_b200 import _lib
    from ceep_b200.fdtd2d import _Desc2S
    import ctypes as C
    assert _lib.lib().ceep2s_desc_size() == C.sizeof(_Desc2S)


def test_config_and_sources_mirror_the_reference():
    from ceep_b200.fdtd2d import (GaussianSource, GridConfig, ModulatedGaussianSource, SimulationConfig,
                                  SimulationMode, SinusoidalSource)
    cfg = SimulationConfig(grid=GridConfig(nx=64, ny=56, dx=1e-3, dy=0.8e-3), mode=SimulationMode.TMZ,
                           total_steps=320)
    assert cfg.dt == float(GOLD["tmz_cpml_dt"])
    name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats = SINGLE2D[1]
    w = GOLD[f"{name}_waveforms"]
    made = []
    for sp in srcs:
        if sp[0] == "gauss":
            made.append(GaussianSource(x=sp[1], y=sp[2], frequency_max=sp[3], amplitude=sp[4], delay_factor=sp[5],
                                       field_component=sp[6]))
        elif sp[0] == "sin":
            made.append(SinusoidalSource(x=sp[1], y=sp[2], frequency=sp[3], amplitude=sp[4], field_component=sp[5]))
    dt = float(GOLD[f"{name}_dt"])
    for k, s in enumerate(made):
        assert np.array_equal(np.array([s.value_at(n, dt) for n in range(steps)]), w[k])
    with pytest.raises(ValueError):
        SimulationConfig(grid=GridConfig(nx=8, ny=8), courant=0.8, total_steps=3)
    m = ModulatedGaussianSource(x=1, y=2, frequency=5e9, bandwidth=4e9)
    assert m.position == (1, 2) and m.component == "Ez"


def test_grid_coefficients_match_the_reference():
    from ceep_b200.fdtd2d import GridConfig, Grid2D, SimulationConfig, SimulationMode
    for case in SINGLE2D:
        name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats = case
        cfg = SimulationConfig(grid=GridConfig(nx=nx, ny=ny, dx=1e-3, dy=0.8e-3),
                               mode=getattr(SimulationMode, mode), total_steps=steps)
        g = Grid2D.__new__(Grid2D)
        g.config = cfg
        g._empty = torch.empty(0)          # the coefficients are formed with torch on this device (CPU here)
        shp = (nx, ny)
        g.eps_r, g.eps_inf, g.mu_r = np.ones(shp), np.ones(shp), np.ones(shp)
        g.sigma_e, g.sigma_m = np.zeros(shp), np.zeros(shp)
        g._version = 0
        for m in mats:
            if m[0] == "circle":
                g.set_material_circle(m[1], m[2], m[3], eps_r=m[4], mu_r=m[5], sigma_e=m[6], sigma_m=m[7])
            else:
                g.set_material_region(m[1], m[2], m[3], m[4], eps_r=m[5], mu_r=m[6], sigma_e=m[7], sigma_m=m[8])
        g._precompute_coefficients()
        for k in ("ca", "cb", "da", "db"):
            assert np.array_equal(getattr(g, "_" + k), GOLD[f"{name}_{k}"]), (name, k)


def test_cpml_coefficients_match_the_oracle():
    from ceep_b200.fdtd2d import cpml_coefficients
    from oracle.fdtd2d_single import cpml_params
    for args in ((8, 1e-3, 1.1e-12, 4, 2.0, 0.05, 1.0), (6, 0.8e-3, 1.3e-12, 3, 1.5, 0.1, 2.0)):
        for a, b in zip(cpml_coefficients(*args), cpml_params(*args)):
            assert np.array_equal(a, b)
