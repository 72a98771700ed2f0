"""The bench's reference arm on CPU: `bench.py --impl reference` runs the reference's own CPU
multigrid cycles on host cores for the stated warm-up and steps and prints one JSON line with the
same metric, unit and config as the GPU arm, marked impl = reference, with its CPU baseline and a
zero-copy e2e block. The timed region it reports (steps x ms_per_step) fits inside its wall time."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libproto_ref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="the reference library is built by build()")
def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--ref-procs", "2"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "MG solves/s" and d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["config"]["workload"].startswith("periodic Poisson multigrid, 256^3")
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    assert cb["cores"] == 2 and cb["timed_s"] > 0
    assert d["steps"] * d["ms_per_step"] / 1000.0 <= d["wall_s"]
    assert abs(d["value"] - 2 * d["steps"] / (cb["timed_s"] * cb["cycles_per_solve"])) < 1e-9 * d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
