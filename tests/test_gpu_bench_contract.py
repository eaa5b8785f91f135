"""The benchmark's JSON line at a small size (8^3 elements, the same operator and code path as the default 64^3 run):
exactly one line, with every key the benchmark contract names -- metric, value, unit, n_gpus, steps, warmup, ms_per_step,
higher_is_better, scaling, vs_baseline, dtype, data, config with the workload, the roofline with bound / achieved / peak /
unit / frac / traffic, the CPU baseline with value / unit / cores / kind / sample, the end-to-end figure with its host-device
bytes, the count of the library's own launches and the clocks seen -- and values that are consistent with one another."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def test_bench_line_carries_the_contract_keys():
    r = subprocess.run([sys.executable, "bench.py", "--size", "8", "--steps", "3", "--warmup", "3", "--no-timeloop"], cwd=ROOT,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
              "dtype", "data", "config", "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] >= 3 and d["higher_is_better"] is True and d["scaling"] == "weak"
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["unit"] == "GDoF/s"
    assert "workload" in d["config"] and "8^3" in d["config"]["workload"]
    rf = d["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in rf, k
    assert rf["bound"] in ("hbm", "tensor") and 0 < rf["frac"] < 1.5 and rf["achieved"] == pytest.approx(rf["frac"] * rf["peak"])
    cb = d["cpu_baseline"]
    for k in ("value", "unit", "cores", "kind", "sample"):
        assert k in cb, k
    assert cb["kind"] in ("port", "reference") and cb["value"] > 0 and cb["cores"] >= 1
    e = d["e2e"]
    for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"):
        assert k in e, k
    dofs = d["config"]["dofs"]
    assert e["h2d_bytes_per_step"] == 3 * 8 * dofs and e["d2h_bytes_per_step"] == 2 * 8 * dofs
    assert 0 < e["value"] <= d["value"] * 1.05
    assert d["gpu_launches"] > 0
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"]
