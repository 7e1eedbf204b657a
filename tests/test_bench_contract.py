"""bench.py's reference arm runs on the host (the reference's own mc_driver_cpu,
compiled unmodified into oracle/_ref) and prints one JSON line with the keys
the benchmark contract asks for.  CPU only; skipped when oracle/_ref is not
built."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ref_lib_path

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_contract_line():
    if ref_lib_path("ref_cpu_bench") is None:
        pytest.skip("oracle/_ref/ref_cpu_bench not built")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "spin-flip attempts/s" and line["unit"] == "attempts/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["warmup"] >= 3 and line["steps"] == 1
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] >= 1 and cpu["value"] == line["value"]
    assert "mc_driver_cpu" in cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "attempts/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in line["config"]


def test_bench_lists_its_workloads():
    r = subprocess.run([sys.executable, "bench.py", "--help"], cwd=REPO, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0
    for w in ("swarm", "batched", "committor", "surrogate", "cnn", "rate", "cluster", "tail"):
        assert w in r.stdout
