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
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--cpu-replicas", "48", "--cpu-sweeps", "300",
                        "--no-reference-gpu"],
                       cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "spin-flip attempts/s" and line["unit"] == "attempts/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["warmup"] >= 3 and line["steps"] == 2 and len(line["step_ms"]) == 2
    assert line["n_gpus"] == 1
    # the same workload config as the GPU arm's line, timed on the CPU sample
    sys.path.insert(0, REPO)
    import bench
    assert line["config"] == bench.CONFIG
    assert line["cpu_config"]["replicas"] == 48 and line["cpu_config"]["sweeps"] == 300
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


def test_cpu_harness_counts_attempts_and_marks_steps():
    """The timing harness reports the attempts the unmodified driver made and
    a timestamp at every output callback, from which bench.py cuts steps."""
    if ref_lib_path("ref_cpu_bench") is None:
        pytest.skip("oracle/_ref/ref_cpu_bench not built")
    sys.path.insert(0, REPO)
    import bench
    run = bench.cpu_reference_run(3, 200, cores=[0])
    assert run["cores"] == 1 and run["attempts"] == 64 * 64 * 3 * 200
    (t0, marks), = run["marks"]
    assert sorted(marks) == list(range(0, 201, bench.CPU_MARK_INT))
    steps = bench.cpu_steps(run, 4)
    assert len(steps) == 4 and all(t >= 0 for t in steps)
    assert abs(sum(steps) - (marks[200] - t0)) < 1e-6


def test_gpus_flag_starts_the_ranks_itself():
    """bench.py --gpus 2 without a launcher starts two ranks (gloo in the dry
    run) and rank 0 alone prints one line with n_gpus 2."""
    r = subprocess.run([sys.executable, "bench.py", "--gpus", "2", "--dry-run", "--steps", "3",
                        "--warmup", "3"], cwd=REPO, capture_output=True, text=True, timeout=600,
                       env={**os.environ, "OMP_NUM_THREADS": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["world_size"] == 2 and line["backend"] == "gloo"
    assert line["steps"] == 3 and line["value"] > 0
