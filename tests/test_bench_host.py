"""Host-side logic of bench.py (no GPU): the benchmark workloads are the
batched L-FTS systems they are named for, the learned start's pair count
rule, and the workload description printed in the JSON line."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_workloads_are_the_named_systems():
    import bench
    assert sorted(bench.WORKLOADS) == ["diblock64", "diblock96"]
    p = bench.workload_params("diblock64")
    assert p["nx"] == [64] * 3 and p["lx"] == [7.3] * 3 and p["chi_n"] == {"A,B": 17.0}
    assert p["langevin"] == {"dt": 0.8, "nbar": 100} and p["saddle"]["tolerance"] == 1e-4
    assert p["distinct_polymers"][0]["blocks"][0]["length"] == 0.5 and bench.WORKLOADS["diblock64"]["replicas"] == 64
    q = bench.workload_params("diblock96")
    assert q["nx"] == [96] * 3 and q["lx"] == [8.0] * 3 and q["chi_n"] == {"A,B": 18.0}
    assert q["langevin"]["nbar"] == 200 and q["distinct_polymers"][0]["blocks"][0]["length"] == 0.4
    assert bench.WORKLOADS["diblock96"]["replicas"] == 16
    # the grid can be overridden, the system stays
    assert bench.workload_params("diblock64", 32)["nx"] == [32] * 3


def test_learned_pair_steps_target_about_1024_pairs():
    import bench
    assert bench.learned_pair_steps(64) == 16
    assert bench.learned_pair_steps(16) == 64
    assert bench.learned_pair_steps(1) == 64      # capped
    assert bench.learned_pair_steps(1024) == 16   # at least 16 steps
    assert bench.learned_pair_steps(24) == 43     # ceil(1024 / 24)


def test_workload_description():
    import bench
    c = bench.workload_config(64, 64)
    assert c["grid"] == [64] * 3 and c["replicas_per_gpu"] == 64 and c["N"] == 90
    assert "64^3" in c["workload"] and "64 replicas" in c["workload"]


def test_cli_names_the_workloads():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0 and "diblock64" in out.stdout and "diblock96" in out.stdout
    bad = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload", "unknown"], capture_output=True,
                         text=True, timeout=120)
    assert bad.returncode != 0
