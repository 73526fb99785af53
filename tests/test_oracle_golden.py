"""The CPU oracle against fixtures produced by the reference implementation.

These pins are what make the oracle trustworthy as the checker for the CUDA
path: every fixture was generated by the reference's own code
(tests/golden/make_golden.py).
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle.fdtd2d import Fdtd2DOracle, run_cpu_oracle
from oracle.fdtd3d import Fdtd3DOracle
from oracle import spectral

SMALL = dict(nx=48, ny=40, dx=0.5e-3, total_steps=260, cpml_thickness=6, frequency=2e9)
SMALL_SRC = [(20, 18), (8, 30), (40, 6)]
SMALL_PRB = [(20, 18), (7, 7), (41, 33), (24, 2)]
STATE_2D = ["ez", "hx", "hy", "psi_hxy_lo", "psi_hxy_hi", "psi_ezx_lo", "psi_ezx_hi",
            "psi_hyx_lo", "psi_hyx_hi", "psi_ezy_lo", "psi_ezy_hi"]


def test_small_2d_fp64_bit_exact():
    g = load_golden("fdtd2d_small_float64")
    o = Fdtd2DOracle(source_positions=SMALL_SRC, probe_positions=SMALL_PRB,
                     eps_r=g["eps_r"], sigma_e=g["sigma_e"], **SMALL)
    assert o.dt == float(g["dt"])
    o.run()
    np.testing.assert_array_equal(o.probe_data, g["probes"])
    for k in STATE_2D:
        np.testing.assert_array_equal(getattr(o, k), g[k], err_msg=k)


def test_small_2d_fp32_reference_close_to_fp64():
    g32, g64 = load_golden("fdtd2d_small_float32"), load_golden("fdtd2d_small_float64")
    assert rel_l2(g32["probes"], g64["probes"]) < 1e-5


def test_cfg1_fp64_bit_exact():
    g = load_golden("fdtd2d_cfg1_float64")
    pos = [tuple(p) for p in g["positions"]]
    x, y = np.meshgrid(np.arange(200), np.arange(200), indexing="ij")
    m = (x - 100) ** 2 + (y - 100) ** 2 <= 40 ** 2
    eps = np.where(m, 40.0, 1.0)
    sig = np.where(m, 0.5, 0.0)
    o = Fdtd2DOracle(200, 200, 0.5e-3, 400, 15, pos, pos, 2e9, eps_r=eps, sigma_e=sig)
    o.run()
    np.testing.assert_array_equal(o.probe_data, g["probes"])
    assert rel_l2(load_golden("fdtd2d_cfg1_float32")["probes"], g["probes"]) < 1e-5


def _ceep_results_case(kind):
    g = load_golden("ceep_results")
    nx = 64
    eps = np.ones((nx, nx)); sig = np.zeros((nx, nx))
    x, y = np.ogrid[:nx, :nx]
    if kind in ("brain", "hemorrhage"):
        m = np.sqrt((x - 32) ** 2 + (y - 32) ** 2) < 20
        eps[m], sig[m] = 50.0, 1.5
    if kind == "hemorrhage":
        m = np.sqrt((x - 40) ** 2 + (y - 37) ** 2) < 10
        eps[m], sig[m] = 60.0, 2.0
    o = Fdtd2DOracle(nx, nx, 0.5e-3, 100, 10, [(32, 32)], [(32, 32)], 2e9, eps_r=eps, sigma_e=sig)
    return o.run()[0, 0], g[kind]


@pytest.mark.parametrize("kind", ["brain", "hemorrhage"])
def test_ceep_results_json(kind):
    out, ref = _ceep_results_case(kind)
    assert rel_l2(out, ref) < 1e-14


def test_ceep_results_empty_prefix():
    # The published 'empty' series came from an older boundary implementation:
    # samples 0-42 agree exactly with the shipped code, the reflection from the
    # boundary reaches the antenna at sample 43 and the series drift apart.
    out, ref = _ceep_results_case("empty")
    assert rel_l2(out[:43], ref[:43]) < 1e-14
    assert rel_l2(out[:48], ref[:48]) < 1e-10


def test_run_cpu_variant():
    g = load_golden("fdtd2d_runcpu")
    out = run_cpu_oracle(40, 36, 0.5e-3, 150, [(10, 12), (30, 20), (19, 30)],
                         [(10, 12), (25, 25), (5, 31)], 2e9, eps_r=g["eps_r"], sigma_e=g["sigma_e"])
    np.testing.assert_array_equal(out, g["probes"])


def test_3d_fp64_bit_exact():
    g = load_golden("fdtd3d_small_float64")
    src = [tuple(p) for p in g["src"]]
    prb = [tuple(p) for p in g["prb"]]
    o = Fdtd3DOracle(20, 20, 20, 1e-3, 70, 4, src, prb, 2e9, eps_r=g["eps_r"], sigma_e=g["sigma_e"],
                     mu_r=g["mu_r"], sigma_m=g["sigma_m"])
    assert o.dt == float(g["dt"])
    o.run()
    np.testing.assert_array_equal(o.probe_data, g["probes"])
    for k in ["ex", "ey", "ez", "hx", "hy", "hz", "psi_hxy_lo", "psi_hxy_hi", "psi_hyx_lo"]:
        np.testing.assert_array_equal(getattr(o, k), g[k], err_msg=k)
    assert o.compute_energy() == float(g["energy"])


def test_dft_matches_reference_monitor():
    g = load_golden("dft_cfg1")
    c = load_golden("fdtd2d_cfg1_float64")
    S = spectral.running_dft(c["probes"], float(c["dt"]), g["frequencies"])
    assert S.shape == (101, 8, 8)
    assert rel_l2(S, g["S"]) < 1e-14


def test_das_and_dmas_match_reference():
    g = load_golden("das_small")
    pos = [tuple(p) for p in g["positions"]]
    das = spectral.das_frequency(g["S"], g["frequencies"], pos, tuple(g["x_range"]), tuple(g["y_range"]),
                                 float(g["dx"]), float(g["eps_bg"]), frequency_range=tuple(g["frange"]))
    assert rel_l2(das, g["das"]) < 1e-12
    dmas = spectral.dmas_frequency(g["S"], g["frequencies"], pos, tuple(g["x_range"]), tuple(g["y_range"]),
                                   float(g["dx"]), float(g["eps_bg"]))
    assert rel_l2(dmas, g["dmas"]) < 1e-12


def test_das_time_matches_reference():
    g = load_golden("das_time_small")
    img = spectral.das_time(g["s"], g["positions"], float(g["frequency"]), int(g["grid_size"]), float(g["dx"]))
    np.testing.assert_allclose(img, g["image"], rtol=1e-13, atol=0)


def test_ade_composition():
    g = load_golden("ade2d_small")
    nx, ny = 44, 40
    lor = g["lor_mask"]
    # the second add_poles() call of the fixture resets pole 0 inside the
    # Lorentz disk, so the Debye pole only lives where the disks do not overlap
    deb = g["deb_mask"] & ~lor
    disp = {"debye": [(np.where(deb, 30.0, 0.0), np.where(deb, 9e-12, 0.0))],
            "lorentz": [(np.where(lor, 5.0, 0.0), np.where(lor, 2 * np.pi * 6e9, 0.0),
                         np.where(lor, 2 * np.pi * 0.5e9, 0.0))]}
    o = Fdtd2DOracle(nx, ny, 0.5e-3, 220, 5, [(14, 20), (30, 12)], [(14, 20), (30, 12), (22, 30)], 2e9,
                     eps_r=g["eps_r"], sigma_e=g["sigma_e"], dispersion=disp)
    o.run()
    assert rel_l2(o.probe_data, g["probes"]) < 1e-13
    assert rel_l2(o.j_deb[0], g["j0"]) < 1e-12
    assert rel_l2(o.j_lor[0], g["j1"]) < 1e-12


def test_brain_phantom_oracle_against_reference():
    """oracle/phantoms.py against BrainPhantom2D (fixed tissue table) and the
    dataset generator's hemorrhage mask, bit for bit."""
    from oracle.phantoms import brain_phantom_maps, hemorrhage_mask
    g = load_golden("brain_phantom")
    k = 0
    while f"case_{k}" in g:
        nx, ny, dx, hx, hy, rad, head = g[f"case_{k}"]
        loc = None if np.isnan(hx) else (hx, hy)
        eps, sig = brain_phantom_maps(int(nx), int(ny), dx, loc, rad, head)
        np.testing.assert_array_equal(eps, g[f"eps_{k}"])
        np.testing.assert_array_equal(sig, g[f"sigma_{k}"])
        np.testing.assert_array_equal(hemorrhage_mask(int(nx), int(ny), dx, loc, rad), g[f"mask_{k}"])
        k += 1
    assert k == 4
