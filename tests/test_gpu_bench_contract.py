"""The benchmark's GPU line (a short run: config 2 only, 3 warm-up steps, 2 timed): one JSON
line with the contract's keys, the device-timed value, the end-to-end figure through the
public API with its host-device bytes, the roofline of the dominant kernel against a
measured peak, the clock record and the library's own launch count."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_has_the_contract_keys():
    r = subprocess.run([sys.executable, "bench.py", "--steps", "2", "--warmup", "3", "--no-adjoint", "--no-config3",
                        "--no-config5", "--no-cpu-baseline", "--no-reference-gpu"],
                       cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "clocks", "gpu_launches"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3 and d["value"] > 0
    assert d["config"]["workload"] and d["scaling"] == "weak"
    e2e = d["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    roof = d["roofline"]
    assert roof["kernel"] == "k_wf_any" and 0 < roof["frac"] <= 1.2
    assert abs(roof["frac"] - roof["achieved"] / roof["peak"]) < 1e-3
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"] and d["gpu_launches"] > 0
