"""bench.py --impl reference on the host cores: the JSON line a caller parses
(rank 0 only; other ranks print nothing and exit 0). Small N so it runs in
about a second; no GPU is needed."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "1",
        "--n", "20000", "--cpu-seconds", "1"]


def run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run(ARGS, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_line():
    r = run({})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "interactions/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0
    assert d["config"]["n"] == 20000 and d["config"]["workload"].startswith("shell N=20000")
    # the reference's accepted nodes over every particle of the same initial state the GPU arm steps from
    assert d["interactions_per_step"] > 20000 and "initial shell" in d["config"]["state"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert "particles walked" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_silent():
    r = run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [x for x in r.stdout.splitlines() if x.startswith("{")]
