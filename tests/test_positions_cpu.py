"""Antenna positions pinned to the reference (fixture tests/golden/positions.npz,
made by make_golden.py from the reference's own code):
``circular_array_positions`` against CircularArray._compute_elements
(src/ceep/antennas/arrays.py:110-143) and ``ring_positions`` against the
dataset generator's circle (scripts/generate_corrected_dataset.py:121-129)."""
import os

import numpy as np

from conftest import ROOT
from ceep_b200.phantoms import circular_array_positions, ring_positions

G = np.load(os.path.join(ROOT, "tests", "golden", "positions.npz"))


def test_circular_array_positions_match_the_reference():
    k = 0
    while f"circular_{k}" in G.files:
        n, rmm, dx, cx, cy, cz = G[f"circular_case_{k}"]
        c = (int(cx), int(cy)) if G[f"circular_{k}"].shape[1] == 2 else (int(cx), int(cy), int(cz))
        got = circular_array_positions(int(n), float(rmm), c, float(dx))
        assert got == [tuple(int(v) for v in p) for p in G[f"circular_{k}"]], k
        k += 1
    assert k >= 6


def test_ring_positions_match_the_dataset_generator():
    k = 0
    while f"dataset_{k}" in G.files:
        nx, n_ant = (int(v) for v in G[f"dataset_case_{k}"])
        got = ring_positions(n_ant, (nx // 2, nx // 2), nx // 3)
        assert got == [tuple(int(v) for v in p) for p in G[f"dataset_{k}"]], k
        k += 1
    assert k >= 5


def test_the_two_circles_differ_where_truncation_is_at_an_ulp():
    """12 antennas, r = 70 cells: r cos(5 pi / 3) is 35 within an ulp, and the
    two formulas truncate it to different cells; each helper matches its own
    reference caller (checked above), so callers must pick the right one."""
    a = circular_array_positions(12, 70.0, (100, 100), 1e-3)
    b = ring_positions(12, (100, 100), 70)
    assert sum(p != q for p, q in zip(a, b)) == 1
