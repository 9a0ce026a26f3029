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


class _FakeSim:
    """Stands in for amk.Simulation in tree_roofline: phase times, FMM
    statistics and the FFMA probe of a tensor-mode p = 7 step."""

    def __init__(self, near_ms, products_ms):
        self.near_ms, self.products_ms = near_ms, products_ms

    def set_profiling(self, on):
        pass

    def reset_phase_times(self):
        pass

    def step(self, n):
        pass

    def synchronize(self):
        pass

    def phase_times(self):
        return {"fmm_m2l_products": (self.products_ms, 1), "fmm_m2l": (2 * self.products_ms, 1),
                "fmm_near": (self.near_ms, 1)}

    def fmm_stats(self):
        return {"order": 7, "m2l_class_pairs": 13_000_000, "m2l_pairs": 13_100_000, "m2l_classes": 29_000,
                "p2p_particle_pairs": 5_000_000_000}

    def measure_fp32_peak(self):
        return 72.0


@pytest.mark.parametrize("near_ms,products_ms,kernel", [(6.7, 3.7, "fmm_p2p32_kernel"),
                                                         (2.0, 3.7, "m2l_class_tc_kernel<7>")])
def test_tree_roofline_reports_the_dominant_kernel(near_ms, products_ms, kernel):
    # the roofline object describes whichever of the near-field pairs and the
    # M2L class products takes longer per launch, and carries the other one
    sys.path.insert(0, ROOT)
    import bench
    over = {"coulomb_method": "fast-multipole", "fast_multipole_order": 7, "precision": "tensor"}
    r = bench.tree_roofline(_FakeSim(near_ms, products_ms), over, 1 << 20)
    assert r["kernel"] == kernel and r["other_kernel"]["kernel"] != kernel
    near = r if kernel == "fmm_p2p32_kernel" else r["other_kernel"]
    assert near["achieved"] == pytest.approx(20.0 * 5e9 / (near_ms * 1e-3) / 1e12)
    assert near["frac"] == pytest.approx(near["achieved"] / 72.0)
    prod = r["other_kernel"] if kernel == "fmm_p2p32_kernel" else r
    assert prod["achieved"] == pytest.approx(2.0 * 120 * 120 * 13e6 / (products_ms * 1e-3) / 1e12)
