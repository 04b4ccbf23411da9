"""The benchmark's JSON contract on the CPU: the reference arm (the oracle
on the host cores) prints one line with every key the driver reads."""
import json
import os
import subprocess
import sys

from conftest import ROOT

REQUIRED = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline",
            "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "uniform", "--order", "2", "--steps", "1", "--warmup", "3", "--ref-budget", "2"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert REQUIRED <= set(d), REQUIRED - set(d)
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 3
    assert d["value"] > 0 and d["unit"] == "cell-updates/s" and d["higher_is_better"] is True
    assert d["dtype"] == "f64" and "workload" in d["config"]
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0


def test_warmup_below_three_is_refused():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--warmup", "2"],
                       cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "warmup" in r.stderr


def test_reference_arm_serving_workload_line():
    """The default workload's CPU arm: the served-ensemble metric, sampled
    on the ensemble's smallest-grid requests of both schemes."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3", "--ref-budget", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert REQUIRED <= set(d), REQUIRED - set(d)
    assert d["metric"] == "FP64 cell-updates/s on 1 B200, batched vs plain; ensemble p50/p99 latency"
    assert d["config"]["requests"] == 256 and d["config"]["steps_per_request"] == 1
    assert "PLM-MC+Rusanov" in d["cpu_baseline"]["sample"] and "WENOZ+Roe" in d["cpu_baseline"]["sample"]
    assert d["value"] > 0


def test_reference_arm_slabs_workload_line():
    """The sharded-shell workload's CPU arm: config 5's scheme and size in
    `config`, strong scaling (one shell however many GPUs)."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "slabs",
                          "--steps", "1", "--warmup", "3", "--ref-budget", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert REQUIRED <= set(d), REQUIRED - set(d)
    assert d["scaling"] == "strong" and d["config"]["cells"] == 6 * 256 * 192 * 192
    assert d["config"]["scheme"]["spatial_order"] == 4 and d["config"]["scheme"]["gravity"] == 1
    assert d["value"] > 0
