"""Per-run records and NVTX phases (ceep_b200.trace) without a GPU."""
import json

from ceep_b200 import trace


class _Solver:
    record_path = None
    run_record = None


def test_phase_is_harmless_without_a_gpu():
    with trace.phase("time_loop"):
        x = 1
    assert x == 1


def test_records_are_stored_and_appended_as_json_lines(tmp_path):
    s = _Solver()
    s.record_path = str(tmp_path / "runs.jsonl")
    r1 = trace.make_record("BatchedFDTD2D", 600 * 600, 800, 16, 0.032)
    trace.emit(s, r1)
    trace.emit(s, trace.make_record("BatchedFDTD3D", 192 ** 3, 1000, 8, 1.0, status=5))
    assert s.run_record["solver"] == "BatchedFDTD3D" and s.run_record["status"] == 5
    lines = [json.loads(l) for l in open(s.record_path)]
    assert len(lines) == 2 and lines[0]["steps"] == 800
    assert abs(lines[0]["gcell_steps_per_s"] - 600 * 600 * 800 * 16 / 0.032 / 1e9) < 1e-3
