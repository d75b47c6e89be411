"""bench.py's reference arm on the CPU (no GPU): the line the driver reads for the
reference's own throughput -- the CPU restatement timed on the host threads, on the same
workload, metric and unit as the GPU arm -- at a small size of each workload."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("args", [["--dx", "0.03"], ["--workload", "tensile_bar3d", "--dx", "0.5"]],
                         ids=["dambreak3d", "tensile_bar3d"])
def test_reference_arm_line(args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "3"] + args,
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "particle-steps/s" and d["higher_is_better"] is True
    assert d["metric"].startswith("particle-steps/s on 1 B200")
    assert d["value"] > 0.0 and d["ms_per_step"] > 0.0
    assert d["config"]["particles"] > 1000
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "CPU restatement" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
