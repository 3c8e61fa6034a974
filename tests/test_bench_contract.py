"""``bench.py --impl reference`` (the CPU arm, no GPU needed) prints one JSON
line with the benchmark contract's keys, on a small flake with a short sample;
ranks other than 0 print nothing and exit 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, "bench.py", "--impl", "reference", "--flake", "2", "--cpu-budget", "1",
       "--steps", "1", "--warmup", "3"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run(CMD, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_line():
    r = _run({"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "sTDA solves/s" and d["unit"] == "solves/s"
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert abs(d["value"] * d["ms_per_step"] - 1e3) < 1e-6 * 1e3
    assert (d["steps"], d["warmup"], d["n_gpus"]) == (1, 3, 1)
    assert d["higher_is_better"] is True and d["scaling"] == "weak"
    assert d["data"] == "synthetic" and d["config"]["workload"] == "flake n=2 (profiling case)"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_are_silent():
    r = _run({"RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
