"""bench.py's reference arm (the CPU port of the reference PA element loop,
timed on the host cores) runs without a GPU and prints the one JSON line of
the bench contract: same metric, unit and direction as the GPU arm, a
cpu_baseline describing the sample, and an e2e block with no host-device
traffic.  Under torchrun only rank 0 works and prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env=None):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    return lines


def test_reference_arm_json_line():
    lines = _run(["--impl", "reference", "--steps", "3", "--warmup", "3"])
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GDOF/s" and d["higher_is_better"] is True
    assert d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_uses_all_host_threads_under_a_launcher_setting():
    # torchrun sets OMP_NUM_THREADS=1 for every rank; the reference arm still uses every usable host thread
    env = dict(os.environ, OMP_NUM_THREADS="1")
    d = json.loads(_run(["--impl", "reference", "--steps", "3", "--warmup", "3"], env=env)[0])
    assert d["cpu_baseline"]["cores"] == len(os.sched_getaffinity(0))
