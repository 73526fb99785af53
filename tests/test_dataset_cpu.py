"""Host logic of the dataset generator (ceep_b200.dataset): seeded draws,
the reference's per-sample metadata schema and step-count formula."""
import numpy as np

from ceep_b200 import dataset as ds


def test_draws_are_seeded_and_follow_the_reference_ranges():
    a, b = ds.draw_samples(200, 0.7, seed=11), ds.draw_samples(200, 0.7, seed=11)
    assert a == b
    assert sum(s.include_hemorrhage for s in a) == int(200 * 0.7)
    for s in a:
        if s.include_hemorrhage:
            assert np.hypot(*s.center_cm) <= 3.0 and 0.3 <= s.radius_cm <= 1.5
        else:
            assert s.center_cm is None
    assert ds.draw_samples(200, 0.7, seed=12) != a


def test_metadata_schema_matches_the_reference():
    # keys written by scripts/generate_corrected_dataset.py:159-177
    spec = ds.SampleSpec(3, True, (1.0, -0.5), 0.8)
    m = ds.sample_metadata(spec, 64, 64, 0.5e-3, 2e9, 16, 2)
    assert set(m) == {"sample_id", "include_hemorrhage", "hemorrhage_params", "simulation_params",
                      "correction_applied", "correction_factor", "meep_validated"}
    assert set(m["hemorrhage_params"]) == {"center_x", "center_y", "radius"}
    assert set(m["simulation_params"]) == {"nx", "ny", "dx", "frequency", "n_antennas", "total_steps"}
    assert ds.sample_metadata(ds.SampleSpec(4, False), 64, 64, 0.5e-3, 2e9, 16, 2)["hemorrhage_params"] is None


def test_reference_step_formula():
    # int(2 * sqrt(2) * nx * dx / c / (1 / (4 f))): 2 steps at the default 64x64, 0.5 mm, 2 GHz
    assert ds.reference_total_steps(64, 0.5e-3, 2e9) == 2
    assert ds.reference_total_steps(600, 0.5e-3, 2e9) == int(2 * np.sqrt(2) * 0.3 / 3e8 * 8e9)


def test_layer_radii_match_the_oracle():
    from oracle.phantoms import layer_radii
    assert ds.layer_radii(9.0) == layer_radii(9.0)
    assert ds.layer_radii(4.0) == layer_radii(4.0)
