"""The benchmark's reference arm on the CPU: `bench.py --impl reference` times
the oracle port of the host path on the host cores and prints one JSON line
with the metric, unit and direction of the default line, a cpu_baseline
that describes the run, and an e2e entry with no host copies.  Under
torchrun only rank 0 works and prints; the other ranks exit 0 silently.
A small lattice keeps the run to about a second."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--sites", "32,16,32", "--steps", "1",
        "--warmup", "0"]


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run(ARGS, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "points/s" and d["higher_is_better"] is True
    assert d["metric"].startswith("points/s rebuild+scatter+gather")
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["config"]["points_per_gpu"] == 32 * 16 * 32
    assert d["config"]["l2"].startswith("inputs smaller than L2")  # 384 KB of positions and velocities


def test_reference_arm_other_ranks_silent():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
