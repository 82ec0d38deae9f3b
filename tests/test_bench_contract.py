"""bench.py's reference arm on CPU: one JSON line on stdout with the keys and
meanings the measurement contract gives it (the oracle port timed on the host
cores, on the same workload, metric and unit as the CUDA arm; no host-device
copies in its end-to-end figure)."""

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _reference_line(workload: str) -> dict:
    out = subprocess.run(
        [sys.executable, "bench.py", "--impl", "reference", "--workload", workload, "--steps", "1", "--warmup", "3"],
        cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("workload", ["dam", "batch"])
def test_reference_arm_line(workload):
    d = _reference_line(workload)
    assert d["impl"] == "reference"
    for key in ("metric", "unit", "config", "dtype", "data"):
        assert isinstance(d[key], (str, dict)) and d[key]
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] >= 3
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["higher_is_better"] is True
    assert isinstance(d["config"]["workload"], str)
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_do_nothing():
    """Under torchrun with N > 1 only rank 0 runs the reference arm and prints
    its line; every other rank exits 0 at once, printing nothing."""
    import os

    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT="29555")
    out = subprocess.run(
        [sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--workload", "dam", "--steps", "1",
         "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
