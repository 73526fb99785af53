"""Dataset generation on the device against the reference's phantom (via the
pinned oracle) and against individual solver runs."""
import json

import numpy as np
import pytest
import torch

from ceep_b200 import dataset as ds
from oracle.phantoms import brain_phantom_maps, hemorrhage_mask

pytestmark = pytest.mark.gpu


def test_device_phantom_maps_match_the_reference_bit_for_bit(cuda_device):
    specs = [ds.SampleSpec(0, True, (2.1, -1.3), 1.2), ds.SampleSpec(1, False),
             ds.SampleSpec(2, True, (-0.4, 0.25), 0.6), ds.SampleSpec(3, True, (0.0, 0.0), 0.3)]
    for nx, ny, dx, head in ((400, 380, 0.5e-3, 9.0), (64, 64, 0.5e-3, 9.0), (90, 70, 1e-3, 4.0)):
        eps, sig, mask = ds.brain_phantom_maps(specs, nx, ny, dx, head, cuda_device)
        for k, s in enumerate(specs):
            loc = s.center_cm if s.include_hemorrhage else None
            e0, s0 = brain_phantom_maps(nx, ny, dx, loc, s.radius_cm, head)
            np.testing.assert_array_equal(eps[k].cpu().numpy(), e0)
            np.testing.assert_array_equal(sig[k].cpu().numpy(), s0)
            np.testing.assert_array_equal(mask[k].cpu().numpy(), hemorrhage_mask(nx, ny, dx, loc, s.radius_cm))


def test_generated_dataset_files_and_values(cuda_device, tmp_path):
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.phantoms import ring_positions
    nx, ny, T, n_ant = 56, 52, 36, 8
    meta = ds.generate_dataset(n_samples=5, output_dir=str(tmp_path), hemorrhage_ratio=0.6, nx=nx, ny=ny,
                               n_ant=n_ant, total_steps=T, seed=4, batch=3, device=cuda_device)
    assert meta["n_samples"] == 5 and json.load(open(tmp_path / "dataset_metadata.json"))["n_samples"] == 5
    specs = ds.draw_samples(5, 0.6, seed=4)
    for spec in specs:
        name = f"sample_{spec.sample_id:06d}"
        S = np.load(tmp_path / "s_matrix" / f"{name}.npy")
        eps = np.load(tmp_path / "eps_map" / f"{name}.npy")
        mask = np.load(tmp_path / "hem_mask" / f"{name}.npy")
        md = json.load(open(tmp_path / "metadata" / f"{name}.json"))
        assert S.shape == (n_ant, n_ant, T) and S.dtype == np.float64
        assert eps.shape == (nx, ny) and mask.shape == (nx, ny)
        assert md["include_hemorrhage"] == spec.include_hemorrhage and md["simulation_params"]["total_steps"] == T
        # one solver run of the same phantom, through the public API
        loc = spec.center_cm if spec.include_hemorrhage else None
        e0, s0 = brain_phantom_maps(nx, ny, 0.5e-3, loc, spec.radius_cm)
        np.testing.assert_array_equal(eps, e0)

        class Maps:
            eps_r, sigma_e = e0, s0

        pos = ring_positions(n_ant, (nx // 2, ny // 2), nx // 3)
        solo = BatchedFDTD2D(nx, ny, 0.5e-3, T, 10, pos, pos, 2e9)
        solo.set_phantom(Maps())
        out = solo.run()
        want = np.array([[out[t][r] for r in range(n_ant)] for t in range(n_ant)]) * ds.CORRECTION_FACTOR
        np.testing.assert_array_equal(S, want)
        assert np.abs(S).max() > 0
