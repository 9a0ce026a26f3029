"""Host side of bench.py on CPU: the reference arm times the reference's own
CPU code without importing this repository's CUDA library, prints the
workload description the GPU arm prints, honours --steps, and carries the
keys the benchmark contract asks for."""
import json
import os
import subprocess
import sys

import pytest

import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

REQUIRED = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
def test_reference_arm_runs_the_reference_without_the_cuda_library():
    code = ("import sys, json; sys.argv = ['bench.py']; import bench; "
            "rc = bench.main(['--impl', 'reference', '--steps', '2', '--warmup', '3', '--ref-sample', '4096']); "
            "print('AMK_IMPORTED', 'amk' in sys.modules); sys.exit(rc)")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    lines = res.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert lines[-1] == "AMK_IMPORTED False"
    for k in REQUIRED:
        assert k in line, k
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 3
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert "4,096" in line["cpu_baseline"]["sample"]
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.tree_config(1 << 20, 1)  # the GPU arm prints exactly this dict
    # value counts the particles actually processed: sample x steps / time
    assert abs(line["value"] - 4096 * 1e3 / line["ms_per_step"]) <= 1e-6 * line["value"]


def test_default_workload_is_the_1m_tree_solver_comparison():
    sys.path.insert(0, ROOT)
    import bench
    assert {"tree1m", "direct65k", "sweep512", "long4m", "kernels"} <= set(bench.WORKLOADS)
    src = open(os.path.join(ROOT, "bench.py")).read()
    assert 'default="tree1m"' in src
    cfg = bench.tree_config(1 << 20, 2)
    assert cfg["n_particles"] == 1 << 20 and cfg["error_budget"] == 1e-5 and "replicas x2" in cfg["parallelism"]
