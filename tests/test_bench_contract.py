"""bench.py's reference arm on the CPU: one JSON line with the fields the
timing contract names, measured on complete circuits of the CPU restatement
(no extrapolation), without loading the engine's library."""

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_complete_measurement():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--qubits", "14",
                          "--depth", "4", "--steps", "2", "--warmup", "1", "--shots", "100"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT,
                         env={**os.environ, "DQSIM_DEBUG_LIB": "1"})
    assert out.returncode == 0, out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.strip() and not ln.startswith("dqsim loaded")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["higher_is_better"] is False and d["unit"] == "s"
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["n_gpus"] == 1
    assert d["config"]["qubits"] == 14
    cpu = d["cpu_baseline"]
    assert cpu["value"] == d["value"] and cpu["kind"] in ("port", "reference") and cpu["cores"] >= 1
    assert "no extrapolation" in cpu["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "dqsim loaded" not in out.stdout  # the engine's library stays out of the CPU arm
