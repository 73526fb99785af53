"""The reference arm of bench.py on the host (no GPU): every workload prints
one JSON line with the contract's keys, or an ``unavailable`` line where the
reference has no such path."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def _check_line(d, metric):
    assert d["impl"] == "reference" and d["metric"] == metric
    assert d["value"] > 0 and d["unit"] == "GCell-steps/s" and d["higher_is_better"] is True
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


@pytest.mark.parametrize("workload", ["adjoint400", "adjoint192"])
def test_reference_arm_adjoint_unavailable(workload):
    d = _bench("--workload", workload)
    assert d["impl"] == "reference" and "unavailable" in d


def test_reference_arm_disk200():
    d = _bench("--workload", "disk200", "--steps", "1", "--warmup", "1", "--cpu-steps", "2")
    _check_line(d, "batched FDTD GCell-steps/s")
    assert d["config"]["workload"] == "disk200" and d["config"]["tx"] == 8


def test_reference_arm_single():
    d = _bench("--workload", "single4096", "--small", "--steps", "1", "--warmup", "1")
    _check_line(d, "FDTD2D (non-batched) GCell-steps/s")
    assert d["config"]["nx"] == 1024


def test_pack_cases_match_their_draws():
    sys.path.insert(0, ROOT)
    import numpy as np
    import bench
    cases = bench._pack_cases(12)
    assert len(cases) == 12
    for k, c in enumerate(cases):
        assert 256 <= c["nx"] <= 768 and c["nx"] % 32 == 0 and 256 <= c["ny"] <= 768
        assert 600 <= c["steps"] <= 1200 and 8 <= c["ntx"] <= 16
        assert c["phantom"] == ("lorentz" if k % 3 == 2 else "head")
    assert bench._pack_cases(12) == cases                      # seeded
    assert np.isclose(cases[0]["ring"], 0.36 * min(cases[0]["nx"], cases[0]["ny"]))


def test_reference_arm_pack():
    d = _bench("--workload", "pack256", "--pack-count", "6", "--steps", "1", "--warmup", "1", "--cpu-steps", "1")
    _check_line(d, "packed uneven batch GCell-steps/s")
    assert d["config"]["phantoms"] == 6 and d["config"]["sampled"] >= 1


@pytest.mark.parametrize("steps", [1, 2])
def test_temporal_block_is_always_applied(steps):
    """`--temporal-block 1` must reach the solver even though the solver's own
    default is two steps per launch; 3D workloads stay at one."""
    sys.path.insert(0, ROOT)
    import bench

    class Solver:
        calls = []

        def set_temporal_block(self, n):
            self.calls.append(n)

    s = Solver()
    assert bench.apply_temporal_block(s, bench.WORKLOADS["head600"], steps) == steps
    assert s.calls == [steps]
    s.calls.clear()
    assert bench.apply_temporal_block(s, bench.WORKLOADS["head192"], steps) == 1
    assert s.calls == []
