"""The reference arm of the benchmark prints the driver's JSON line: complete FP64 runs of the reference's own GPU
backend on the benchmark LP (value, e2e) and one complete run of its CPU backend (cpu_baseline). On a machine
without a GPU the reference's GPU backend cannot run, and the arm prints its `unavailable` line instead."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = ROOT / "oracle" / "_ref" / "pdhg"


@pytest.mark.skipif(not REF.exists(), reason="oracle/_ref/pdhg not built (make -C oracle ref)")
def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup",
                          "0", "--no-cpu-baseline"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # no GPU here: the reference GPU backend failed to start
        assert "GPU backend failed" in d["unavailable"]
        return
    assert d["unit"] == "s" and d["higher_is_better"] is False and d["dtype"] == "fp64"
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["e2e"]["value"] >= d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["run"]["statuses"] == ["near_optimal"] and d["run"]["iterations"] == [80448]
    assert d["config"]["m"] == 200_000 and d["config"]["n"] == 500_000
