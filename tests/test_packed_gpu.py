"""Packed multi-phantom launch: every phantom's result equals its own
single-grid run bit for bit, across uneven sizes, step counts, TX counts
(several lane widths and TX groups) and dispersion models."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle.fdtd2d import Fdtd2DOracle

pytestmark = pytest.mark.gpu

SPECS = [
    # nx, ny, steps, ntx, n, kind
    (64, 48, 90, 3, 6, "none"),
    (96, 80, 120, 8, 8, "debye"),
    (72, 72, 60, 16, 6, "lorentz2"),
    (56, 90, 110, 12, 5, "debye+lorentz"),
    (48, 48, 75, 37, 4, "none"),           # two TX groups of 32
    (80, 64, 120, 5, 7, "debye2"),
]


def _make(spec, seed):
    from ceep_b200 import BatchedFDTD2D
    nx, ny, T, ntx, n, kind = spec
    rng = np.random.default_rng(seed)
    src = [(int(rng.integers(n + 1, nx - n - 1)), int(rng.integers(n + 1, ny - n - 1))) for _ in range(ntx)]
    prb = src[:3] + [(nx // 2, ny // 2)]
    x, y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    m = (x - nx // 2) ** 2 + (y - ny // 2) ** 2 <= (min(nx, ny) // 4) ** 2
    eps, sig = np.where(m, 5.0 + rng.random(), 1.0), np.where(m, 0.3, 0.0)
    deb = lambda: (np.where(m, rng.uniform(10, 40), 0.0), np.where(m, rng.uniform(5e-12, 15e-12), 0.0))
    lor = lambda: (np.where(m, rng.uniform(1, 6), 0.0), np.where(m, 2 * np.pi * rng.uniform(2e9, 15e9), 0.0),
                   np.where(m, 2 * np.pi * rng.uniform(0.1e9, 1e9), 0.0))
    disp = {"none": ([], []), "debye": ([deb()], []), "lorentz2": ([], [lor(), lor()]),
            "debye+lorentz": ([deb()], [lor()]), "debye2": ([deb(), deb()], [])}[kind]
    s = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, src, prb, 2e9)
    s._eps_r[:], s._sigma_e[:] = eps, sig
    if kind != "none":
        s.set_dispersion(debye=disp[0], lorentz=disp[1])
    return s, (eps, sig, disp)


def test_packed_equals_individual_runs(cuda_device):
    from ceep_b200.packed import PackedBatch2D
    solo = []
    for k, spec in enumerate(SPECS):
        s, _ = _make(spec, k)
        s.set_rows_per_block(12)
        s.run()
        solo.append(s.probe_data.clone())
    packed = [_make(spec, k)[0] for k, spec in enumerate(SPECS)]
    pk = PackedBatch2D(packed, rows=12)
    pk.run()
    for a, s in zip(solo, packed):
        assert torch.equal(a, s.probe_data)
    assert pk.tiles_at(0) > pk.tiles_at(pk.max_steps - 1)    # finished phantoms drop out


def test_packed_against_oracle_and_autotune(cuda_device):
    from ceep_b200.packed import PackedBatch2D
    made = [_make(spec, 10 + k) for k, spec in enumerate(SPECS[:4])]
    pk = PackedBatch2D([m[0] for m in made])
    timings = pk.autotune(candidates=(8, 16, 24), probe_steps=20)
    pks = (0, 1) if pk.classes > 1 else (0,)
    assert set(timings) == {(tb, r, c) for tb in (1, 2) for r in (8, 16, 24) for c in pks}
    assert (pk.temporal_block, pk.rows, pk.packing) in timings
    results = pk.run()
    for (s, (eps, sig, disp)), res, spec in zip(made, results, SPECS):
        o = Fdtd2DOracle(s.nx, s.ny, 0.5e-3, s.total_steps, s.cpml_n, s.source_positions, s.probe_positions,
                         2e9, eps_r=eps, sigma_e=sig, dispersion={"debye": disp[0], "lorentz": disp[1]})
        o.run()
        got = np.array([[res[b][p] for p in range(len(s.probe_positions))] for b in range(s.batch)])
        assert rel_l2(got, o.probe_data) < 1e-4, spec


def test_packed_two_steps_per_launch_equals_individual_runs(cuda_device):
    """temporal_block=2: every running phantom advances two steps per launch
    (the 75-step phantom takes its last step alone); probe series and final
    fields equal each phantom's own run bit for bit."""
    from ceep_b200.packed import PackedBatch2D
    solo = []
    for k, spec in enumerate(SPECS):
        s, _ = _make(spec, 20 + k)
        s.set_rows_per_block(12)
        s.run()
        solo.append((s.probe_data.clone(), s.ez.clone(), s.hx.clone()))
    packed = [_make(spec, 20 + k)[0] for k, spec in enumerate(SPECS)]
    pk = PackedBatch2D(packed, rows=12, temporal_block=2)
    pk.run()
    for (pd, ez, hx), s in zip(solo, packed):
        assert torch.equal(pd, s.probe_data)
        assert torch.equal(ez, s.ez) and torch.equal(hx, s.hx)
    # a run in two halves (even bounds) gives the same
    pk.reset()
    pk.advance(0, 40)
    pk.advance(40)
    for (pd, ez, hx), s in zip(solo, packed):
        assert torch.equal(pd, s.probe_data) and torch.equal(ez, s.ez)


@pytest.mark.parametrize("tblock", [1, 2])
def test_concurrent_class_chains_equal_individual_runs(cuda_device, tblock):
    """packing=1: each class (lane width x ADE shape) runs its launch chain on
    its own stream; probe series and fields equal each phantom's own run bit
    for bit, with and without graph capture."""
    from ceep_b200.packed import PackedBatch2D
    solo = []
    for k, spec in enumerate(SPECS):
        s, _ = _make(spec, 30 + k)
        s.set_rows_per_block(12)
        s.set_temporal_block(tblock)
        s.run()
        solo.append((s.probe_data.clone(), s.ez.clone()))
    for use_graph in (True, False):
        packed = [_make(spec, 30 + k)[0] for k, spec in enumerate(SPECS)]
        pk = PackedBatch2D(packed, rows=12, temporal_block=tblock, packing=1, use_graph=use_graph)
        assert pk.classes > 1
        pk.run()
        for (pd, ez), s in zip(solo, packed):
            assert torch.equal(pd, s.probe_data) and torch.equal(ez, s.ez)
