"""bench.py's reference arm (the reference's own CPU library on the host cores) keeps the JSON-line
contract, on a small seeded case, without a GPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3",
       "--scale", "0.05", "--ref-step-seconds", "0.2"]


def _run(env_extra=None):
    env = dict(os.environ, **(env_extra or {}))
    return subprocess.run(CMD, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_json_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "pts/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 3
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "pts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("batched_uneven")
    # the same config object as the GPU arm's line (bench.run_config), parallelism included
    assert d["config"]["parallelism"] == "shots x1 (weak)"
    assert "shots at evenly spaced ranks" in d["cpu_baseline"]["sample"]


def test_reference_arm_other_ranks_do_no_work():
    """Under torchrun only rank 0 runs the reference arm and prints; the others exit 0 at once."""
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [x for x in r.stdout.splitlines() if x.startswith("{")]
