"""The non-batched 2D oracle (TMz / TEz, CFS-CPML, PEC, Mur) against the
reference's own FDTD2D run (tests/golden/single2d.npz), and host-side checks
of the drop-in API that need no GPU."""
import os
import sys

import numpy as np
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
