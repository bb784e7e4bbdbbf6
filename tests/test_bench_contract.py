"""bench.py's reference arm on CPU: one JSON line with the contract's keys,
the metric (the GPU arm's string), unit and direction, e2e carrying zero transfer
bytes, and a cpu_baseline describing the run (no GPU needed)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "h2-1k", "--steps", "1", "--warmup", "1", "--cpu-seconds", "2"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "cells/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == "h2-1k" and d["value"] > 0
    assert d["metric"] == "cells/s per ΔT at relTol 1e-4 (h2-1k, R34)"
    assert d["e2e"] == {"value": d["value"], "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]


def test_both_arms_print_the_same_metric():
    """The driver pairs the GPU arm's line with the reference arm's by the metric
    string: every JSON line bench.py builds takes it from metric_name()."""
    import ast
    sys.path.insert(0, ROOT)
    import bench
    src = open(os.path.join(ROOT, "bench.py")).read()
    metrics = [kv for node in ast.walk(ast.parse(src)) if isinstance(node, ast.Dict)
               for kv in zip(node.keys, node.values)
               if isinstance(kv[0], ast.Constant) and kv[0].value == "metric"]
    assert len(metrics) == 2
    for _, v in metrics:
        assert isinstance(v, ast.Call) and getattr(v.func, "id", None) == "metric_name", ast.dump(v)
    assert bench.metric_name("gri-bimodal-1M", 34) == "cells/s per ΔT at relTol 1e-4 (gri-bimodal-1M, R34)"
    # the default workload is the 1M-cell bimodal batch
    sys.argv = ["bench.py"]
    assert bench.parse().workload == "gri-bimodal-1M"
