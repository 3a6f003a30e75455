"""bench.py's reference arm (CPU only: the reference's own solver on the host
cores) keeps the JSON contract: one line with the metric, value, unit,
impl = reference, a cpu_baseline describing the run (with the as-shipped FP32
figure beside the FP64 one) and an e2e object with no host-device bytes."""
import json
import os
import subprocess
import sys

import pytest

from oracle import reference

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args):
    proc = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), *args], capture_output=True, text=True,
                          timeout=900, cwd=REPO)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, proc.stdout[-2000:]
    return json.loads(lines[0])


@pytest.mark.skipif(not (reference.available("f64") and reference.available("f32")),
                    reason="oracle/_ref/ref_f64 and ref_f32 not built")
def test_reference_arm_line():
    d = run_bench("--impl", "reference", "--workload", "straight", "--steps", "1", "--warmup", "0",
                  "--ref-threads", "1")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["value"] > 0
    assert d["config"]["workload"] == "straight_channel_200x100_fou" and d["config"]["converged"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] == 1
    assert cb["as_shipped_fp32"]["value"] > 0 and cb["as_shipped_fp32"]["converged"]
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_thermal_is_unavailable():
    d = run_bench("--impl", "reference", "--workload", "thermal")
    assert d["impl"] == "reference" and "AMGCL" in d["unavailable"]
