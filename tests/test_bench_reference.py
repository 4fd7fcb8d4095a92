"""bench.py's reference arm on CPU: the oracle timed on the host cores (spawned copies)
prints one JSON line with the contract's keys; under torchrun a rank other than 0 exits
without work or output."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = [sys.executable, "bench.py", "--impl", "reference", "--workload", "dipole_2d", "--steps", "1", "--warmup",
        "0", "--time-steps", "4"]


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run(ARGS, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    j = json.loads(lines[0])
    assert j["impl"] == "reference" and j["unit"] == "Gcell/s" and j["higher_is_better"] is True
    assert j["value"] > 0 and j["steps"] == 1 and j["warmup"] == 0
    cb = j["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == j["value"]
    assert j["e2e"] == {"value": j["value"], "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_output():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = subprocess.run(ARGS, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
