"""bench.py's reference arm on the CPU: one bench step per load step of the
path, so --steps equal to the number of load steps times one full path and
the line's value is that measured path (no extrapolation)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.timeout(600)
def test_reference_arm_times_the_full_path():
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--grid", "8", "--load-steps", "3",
           "--steps", "3", "--warmup", "1", "--cpu-threads", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 3 and d["warmup"] == 1
    # value = the three timed load steps = one full path; ms_per_step is per load step
    assert d["value"] == pytest.approx(3 * d["ms_per_step"] / 1e3, rel=1e-12)
    assert "measured time of the full 3-step path" in d["cpu_baseline"]["sample"]
    assert "all converged: True" in d["cpu_baseline"]["sample"]
    assert d["e2e"]["value"] == d["value"]


@pytest.mark.timeout(600)
def test_reference_arm_with_fewer_steps_still_times_a_full_path():
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--grid", "8", "--load-steps", "4",
           "--steps", "2", "--warmup", "1", "--cpu-threads", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert d["steps"] == 2 and d["load_steps_timed"] == 4
    assert "4 load steps timed" in d["cpu_baseline"]["sample"]
    assert "measured time of the full 4-step path" in d["cpu_baseline"]["sample"]
    assert d["value"] == pytest.approx(4 * d["ms_per_step"] / 1e3, rel=1e-12)
