"""Two steps per launch (temporal block of two) against one step per launch:
the same arithmetic, so the probe series and the final state must agree bit
for bit, across lane widths, TX groups, ADE models, CPML sizes, odd step
counts (the last step runs alone) and sources/probes on tile edges."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

CASES = [
    # nx, ny, steps, ntx, cpml, kind
    (60, 52, 41, 16, 6, "debye"),
    (150, 40, 30, 3, 5, "none"),          # 1 float4 per cell: 126-column tiles, two across
    (70, 90, 24, 37, 7, "lorentz2"),      # two TX groups of 32
    (200, 180, 30, 8, 10, "debye+lorentz"),  # interior tiles take the plain path
    (64, 64, 19, 12, 0, "debye"),          # no CPML
    (96, 72, 26, 4, 8, "lorentz"),
    (300, 120, 24, 4, 8, "debye"),         # 1 float4 per cell with interior tiles (their deep ring)
    (160, 140, 20, 40, 6, "debye"),        # 8 float4 per cell, two TX groups, interior tiles
]


def _solver(spec, seed, tblock):
    from ceep_b200 import BatchedFDTD2D
    nx, ny, T, ntx, n, kind = spec
    rng = np.random.default_rng(seed)
    lo = max(n + 1, 1)
    # sources/probes anywhere off the edges, including inside the PML and on
    # columns next to tile boundaries (multiples of the tile width minus 2)
    cols = [c for c in (29, 30, 31, 61, 62, 125, 126, 127) if lo <= c < nx - 1]
    src = []
    for k in range(ntx):
        x = int(rng.choice(cols)) if (k % 3 == 0 and cols) else int(rng.integers(1, nx - 1))
        src.append((x, int(rng.integers(1, ny - 1))))
    prb = src[:4] + [(nx // 2, ny // 2), (1, 1), (nx - 2, ny - 2)]
    x, y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    m = (x - nx // 2) ** 2 + (y - ny // 2) ** 2 <= (min(nx, ny) // 4) ** 2
    s = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, src, prb, 2e9, temporal_block=tblock)
    s._eps_r[:] = np.where(m, 5.0 + rng.random(), 1.0)
    s._sigma_e[:] = np.where(m, 0.3, 0.0)
    deb = lambda: (np.where(m, rng.uniform(10, 40), 0.0), np.where(m, rng.uniform(5e-12, 15e-12), 0.0))
    lor = lambda: (np.where(m, rng.uniform(1, 6), 0.0), np.where(m, 2 * np.pi * rng.uniform(2e9, 15e9), 0.0),
                   np.where(m, 2 * np.pi * rng.uniform(0.1e9, 1e9), 0.0))
    d = {"none": ([], []), "debye": ([deb()], []), "lorentz": ([], [lor()]), "lorentz2": ([], [lor(), lor()]),
         "debye+lorentz": ([deb()], [lor()])}[kind]
    if kind != "none":
        s.set_dispersion(debye=d[0], lorentz=d[1])
    return s


@pytest.mark.parametrize("spec", CASES, ids=[f"{c[0]}x{c[1]}-{c[3]}tx-{c[5]}" for c in CASES])
def test_two_step_launch_matches_one_step(cuda_device, spec):
    ref = _solver(spec, 7, 1)
    two = _solver(spec, 7, 2)
    ref.run()
    two.run()
    assert two.launches() == (spec[2] + 1) // 2 and ref.launches() == spec[2]
    rel = lambda a, b: float((a - b).norm() / max(float(b.norm()), 1e-30))
    for name in ("probe_data", "ez", "hx", "hy"):
        a, b = getattr(two, name), getattr(ref, name)
        assert torch.isfinite(a).all()
        assert rel(a, b) < 1e-6, (name, rel(a, b))
    # the ping-pong state is also equal (ADE currents, CPML psi)
    c2, c1 = two._cur(), ref._cur()
    for a, b in ((two._psi_ezx[c2], ref._psi_ezx[c1]), (two._psi_hy[c2], ref._psi_hy[c1])):
        assert rel(a, b) < 1e-6
    if two._j is not None:
        assert rel(two._j[c2], ref._j[c1]) < 1e-6
    bitwise = torch.equal(two.probe_data, ref.probe_data) and torch.equal(two.ez, ref.ez)
    print(f"{spec}: bitwise equal = {bitwise}")


def test_two_step_continues_like_one_step(cuda_device):
    """A second run() continues the simulation (the reference's semantics);
    the ping-pong parity after an odd number of launches is tracked."""
    spec = (60, 52, 21, 16, 6, "debye")
    ref, two = _solver(spec, 3, 1), _solver(spec, 3, 2)
    for s in (ref, two):
        s.run()
        s.run()
    assert float((two.ez - ref.ez).norm() / ref.ez.norm()) < 1e-6
