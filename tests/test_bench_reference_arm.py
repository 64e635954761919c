"""`bench.py --impl reference` on the host: the reference's own A11 kernel
(oracle/_ref) timed on a small mesh prints the benchmark's JSON line, and
ranks other than 0 exit without work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], env=env, cwd=ROOT,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_line(reference_kernels):
    r = run_bench({}, "--impl", "reference", "--size", "6", "--steps", "3", "--warmup", "1")
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GDoF/s" and d["higher_is_better"] is True
    assert d["metric"] == "A11 MF apply GDoF/s (FP64, 6^3 Q2 deformed mesh)"
    assert d["steps"] == 3 and d["warmup"] == 1 and d["value"] > 0.0
    assert d["config"]["dofs"] == 3 * 13 ** 3 and d["config"]["elements"] == 216
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and 1 <= cb["cores"] <= os.cpu_count()
    assert d["e2e"] == {"value": d["value"], "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = run_bench({"RANK": "1", "WORLD_SIZE": "2"}, "--impl", "reference", "--size", "6", "--steps", "3")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
