"""The reference arm of bench.py for the extra workloads, on CPU: ``--impl reference`` prints one
JSON line with the contract's keys (or its ``unavailable`` line) and never needs a GPU."""

import json
import subprocess
import sys

from conftest import ROOT


def _reference_line(*args) -> dict:
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", *args],
                         cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [line for line in out.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_terrain_reference_arm_is_unavailable_with_a_reason():
    line = _reference_line("--workload", "terrain")
    assert line["impl"] == "reference" and "unavailable" in line and line["unavailable"]


def test_box3d_small_reference_arm_reports_the_oracle_baseline():
    line = _reference_line("--workload", "box3d-small")
    assert line["impl"] == "reference" and line["metric"] == "jacobian_entries_per_second"
    assert line["value"] > 0 and line["unit"] == "entries/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "entries/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["rows"] == 4000 and line["config"]["cells"] == 36000
