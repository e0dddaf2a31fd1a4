"""bench.py's reference arm runs on the host cores, so its JSON line is
checked here on CPU: the keys and units the driver reads, and the
metric it shares with the B200 arm."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_json_line():
    """A 64^3 run of the arm (the default, 512^3, takes minutes of CPU)."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--n", "64"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Mpts*steps/s at 64^3 NS+ACDI (fp64 form)"
    assert d["config"]["n"] == 64
    assert d["unit"] == "Mpts*steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["n_gpus"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["config"]["workload"]


def test_default_workload_is_the_headline_config():
    sys.path.insert(0, ROOT)
    import bench
    a = bench.parse([])
    assert (a.n, a.precision, a.ns_only, a.steps >= 1, a.warmup >= 3) == (512, "fp64", False, True, True)
    assert bench.metric_name(a.n, not a.ns_only, a.precision) == bench.METRIC
    assert bench.METRIC.startswith("Mpts*steps/s at 512^3 NS+ACDI")
