"""bench.py's reference arm on the CPU: one JSON line with the keys of the bench contract, on
the same metric, unit and workload as the B200 arm; ranks other than 0 print nothing."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run(args, env=None):
    return subprocess.run([sys.executable, "bench.py", *args], cwd=ROOT, capture_output=True, text=True,
                          timeout=600, env={**os.environ, **(env or {})})


def test_reference_arm_prints_one_contract_line():
    import bench
    r = run(["--impl", "reference", "--steps", "1", "--warmup", "3", "--particles", "8192"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "particles/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["workload"].startswith("AR-8")


def test_reference_arm_is_silent_on_other_ranks():
    r = run(["--impl", "reference", "--steps", "1", "--warmup", "3", "--particles", "8192"],
            env={"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0 and not r.stdout.strip()
