"""bench.py's reference arm on CPU: the reference package itself (installed under
baseline/_ref) timed on the host cores prints one JSON line with the contract's keys,
without importing beamz_b200 in any of its processes; under torchrun a rank other than 0
exits without work or output."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--workload", "dipole_2d", "--steps", "1", "--warmup", "0", "--time-steps", "4"]
HAVE_REF = os.path.exists(os.path.join(ROOT, "baseline", "_ref", "beamz", "simulation", "fdtd.py"))
# run bench.py as __main__, then report which beamz_b200 modules the parent process holds
RUNNER = ("import runpy, sys; sys.argv = ['bench.py'] + sys.argv[1:]; "
          "runpy.run_path('bench.py', run_name='__main__'); "
          "print('LOADED ' + ','.join(m for m in sys.modules if m.startswith('beamz_b200')))")


def _run(env=None):
    return subprocess.run([sys.executable, "-c", RUNNER, *ARGS], cwd=ROOT, capture_output=True, text=True,
                          timeout=600, env=env)


@pytest.mark.skipif(not HAVE_REF, reason="the reference is not installed under baseline/_ref")
def test_reference_arm_prints_one_contract_line():
    out = _run()
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    j = json.loads(lines[0])
    assert j["impl"] == "reference" and j["unit"] == "Gcell/s" and j["higher_is_better"] is True
    assert j["value"] > 0 and j["steps"] == 1 and j["warmup"] == 0
    assert j["config"]["grid"] == [400, 400] and j["config"]["time_steps"] == 4
    cb = j["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == j["value"]
    assert j["e2e"] == {"value": j["value"], "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    loaded = [ln for ln in out.stdout.splitlines() if ln.startswith("LOADED")]
    assert loaded == ["LOADED "], loaded


def test_reference_arm_without_install_prints_unavailable(tmp_path):
    """With no reference installed the arm prints its one-line `unavailable` record."""
    import shutil

    for name in ("bench.py",):
        shutil.copy(os.path.join(ROOT, name), tmp_path / name)
    shutil.copytree(os.path.join(ROOT, "beamz_b200"), tmp_path / "beamz_b200",
                    ignore=shutil.ignore_patterns("*.so", "_build", "__pycache__"))
    out = subprocess.run([sys.executable, "bench.py", *ARGS], cwd=tmp_path, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    j = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][0])
    assert j["impl"] == "reference" and "unavailable" in j


def test_reference_arm_other_ranks_exit_without_output():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = _run(env)
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
