"""The benchmark's reference arm (``bench.py --impl reference``) on the host:
it times the reference's host step sequence (the oracle port) and prints one
JSON line with the benchmark's keys; under several ranks only rank 0 runs it.
Small configurations, CPU only."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(args, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [ln for ln in out.stdout.splitlines() if ln.startswith("{")]


def check_line(line):
    d = json.loads(line)
    assert d["impl"] == "reference"
    assert d["unit"] == "ms" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["ms_per_step"] == d["value"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    return d


def test_reference_arm_cube_line():
    lines = run_bench(["--impl", "reference", "--ng", "32", "--ranks", "4", "--steps", "2", "--warmup", "1"])
    assert len(lines) == 1
    d = check_line(lines[0])
    assert d["config"]["ng"] == 32 and d["config"]["world_size"] == 4 and d["config"]["dims"] == [2, 2, 1]
    assert d["steps"] == 2


def test_reference_arm_batch_line():
    lines = run_bench(["--impl", "reference", "--workload", "batch", "--batch-cubes", "4", "--batch-big", "0",
                       "--steps", "1", "--warmup", "1"])
    assert len(lines) == 1
    d = check_line(lines[0])
    assert d["config"]["boxes"] == 4


def test_reference_arm_other_ranks_print_nothing():
    """Launched under several ranks, ranks other than 0 exit 0 without work."""
    lines = run_bench(["--impl", "reference", "--ng", "32", "--ranks", "4", "--steps", "1", "--warmup", "1"],
                      {"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert lines == []
