"""bench.py's reference arm (the oracle port on the host cores): one JSON line
with the metric, the arm's own cpu_baseline and an e2e of zero copies, on
rank 0 only; the other ranks exit 0 without work.  Runs on a small sample so
the CPU suite stays quick."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_arm(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2" if rank else "1", LOCAL_RANK=str(rank))
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                           "--cpu-sample", "24x16"], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=600)


def test_reference_arm_prints_one_contract_line():
    r = run_arm(0)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0.0 and line["unit"] == "cells/s" and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"] == "eddy_1440x1080x75"


def test_reference_arm_other_ranks_exit_quietly():
    r = run_arm(1)
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
