"""The reference arm of bench.py runs on the host cores alone: its JSON line carries the
contract's keys, and ranks other than 0 print nothing."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(env_extra):
    env = dict(os.environ, **env_extra)
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                          "--ref-budget", "1"], capture_output=True, text=True, env=env,
                         timeout=600, check=True)
    return [ln for ln in out.stdout.splitlines() if ln.strip()]


def test_reference_arm_json_line():
    lines = _bench({})
    line = json.loads(lines[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "LJ particle-steps/s" and line["unit"] == "particle-steps/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert "vec SoA twin" in line["cpu_baseline"]["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "particle-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_are_silent():
    assert _bench({"RANK": "1", "WORLD_SIZE": "2"}) == []
