#!/usr/bin/env python
"""Benchmark of the B200 particle path; prints ONE JSON line on rank 0.

Default workload ``tree1m`` -- the 1M-particle solver comparison: N =
1,048,576 positrons in a Gaussian cloud (sigma 1e-4 x 1e-4 x 3e-4 m, numpy
default_rng(42)), 5 K Maxwellian velocities, b0 = 1 T, trap_voltage = 10 V,
z0 = rho0 = 0.01 m, dt from the reference's rule (8.931e-12 s), cooling and
annihilation off. One bench step = one simulation step of the whole cloud
(Coulomb force -> Boris push). Every method (all-pairs, Barnes-Hut theta 0.7,
FMM p = 4/6/7/8 at theta 0.5, learned p = 2 + MLP) is audited against the
FP64 exact sum on 4,096 evenly spaced particles and timed; ``value`` is the
fastest method whose RMS relative force error is <= 1e-5, timed for exactly
``--steps`` steps after ``--warmup`` untimed ones. The same line carries every
method's error and time, the learned / plain p = 6 ratio and the batched /
one-at-a-time ratio of the 512-instance sweep (measured in the same run).

``value`` is particle-steps/s with the state resident in HBM (device-timed
with CUDA events on the library's stream, L2 flushed by a 256 MiB write
between steps, the flush outside the per-step events). ``e2e`` is the same
metric through the C ABI with host buffers: every step uploads x, v from
pinned host memory (amk_update_state), steps, and reads x, v and the alive
flags back (amk_get_particles).

``--impl reference`` times the reference's own CPU code on the host cores:
its FMM (fast-multipole.cc, compiled from the reference sources into
oracle/_ref) at p = 6, theta = 0.5 -- the reference method nearest the 1e-5
error bar -- plus the FP64 Boris push, for whole steps on a bounded sample of
the same cloud (its first 65,536 particles). Nothing of this repository's
CUDA library is imported on that arm.

Other workloads: ``direct65k`` (65,536-particle all-pairs run),
``sweep512`` (the 512-instance batched sweep, partitioned across ranks by a
cost model under torchrun) and ``long4m`` (4,194,304 particles with cooling
and annihilation, learned p = 2 with fallback against plain p = 6, FP64
energy drift every 100 steps).

Multi-GPU: a single instance does not shard (replicas only; ``value`` sums
the replicas over the slowest rank's time); the sweep shards by instance.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "antimatter-kernel_b200"))

METRIC = "particle-steps/s at ≤1e-5 force err vs FP64 direct: learned/batched vs plain"
UNIT = "particle-steps/s"
E = 1.602176634e-19
KB = 1.380649e-23
MASS = {0: 1.67262192369e-27, 1: 9.1093837015e-31, 3: 9.1093837015e-31, 4: 1.67262192369e-27}
ERROR_BUDGET = 1e-5
FLUSH_BYTES = 256 * 1024 * 1024


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.rows = []
        self.proc = None
        self.device_index = device_index

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for k, name in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


# ------------------------------------------------------------------ helpers
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_nccl(world, local):
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))


def finish_dist(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def max_over_ranks(value, world, device):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _dp(ptr):
    return C.cast(C.c_void_p(ptr), C.POINTER(C.c_double))


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_lib as O
    return O


class Flusher:
    """Writes 256 MiB (twice the L2) on the library's stream between steps."""

    def __init__(self, device, stream):
        import torch
        self.torch = torch
        self.buf = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=device)
        self.stream = stream
        self.k = 0

    def __call__(self):
        with self.torch.cuda.stream(self.stream):
            self.buf.fill_(float(self.k))
        self.k += 1


def timed_steps(sim, stream, flusher, k, step_fn=None):
    """k steps, CUDA events around each (on the library's stream), L2 flushed
    between steps outside the events. Returns the summed milliseconds."""
    import torch
    step_fn = step_fn or (lambda: sim.step(1))
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
    for i in range(k):
        starts[i].record(stream)
        step_fn()
        ends[i].record(stream)
        flusher()
    torch.cuda.synchronize()
    return sum(s.elapsed_time(e) for s, e in zip(starts, ends))


def e2e_through_abi(sim, stream, n, steps, step_fn=None):
    """`steps` steps through the C ABI with pinned host buffers: upload x, v,
    step, read x, v and alive back, every step. Returns (ms, h2d, d2h)."""
    import torch
    import amk
    L = amk.lib()
    step_fn = step_fn or (lambda: sim.step(1))
    order = ("x", "y", "z", "vx", "vy", "vz")
    host = {k: torch.empty(n, dtype=torch.float64, pin_memory=True) for k in order}
    alive = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    ptr = {k: v.data_ptr() for k, v in host.items()}
    alive_p = C.cast(C.c_void_p(alive.data_ptr()), C.POINTER(C.c_uint8))
    amk.check(L.amk_get_particles(sim.handle, *[_dp(ptr[k]) for k in order], alive_p))
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        sim.update_state(*[ptr[k] for k in order])
        step_fn()
        amk.check(L.amk_get_particles(sim.handle, *[_dp(ptr[k]) for k in order], alive_p))
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1), 6 * 8 * n, 6 * 8 * n + n


# ================================================================== tree1m
TREE_METHODS = [
    ("allpairs", dict(coulomb_method="allpairs")),
    ("barnes-hut theta=0.7", dict(coulomb_method="barnes-hut", barnes_hut_theta=0.7)),
    ("barnes-hut theta=0.7 tensor", dict(coulomb_method="barnes-hut", barnes_hut_theta=0.7, precision="tensor")),
    ("fmm p=2 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=2, fast_multipole_theta=0.5)),
    ("fmm p=4 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=4, fast_multipole_theta=0.5)),
    ("fmm p=6 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=6, fast_multipole_theta=0.5)),
    ("fmm p=7 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=7, fast_multipole_theta=0.5)),
    ("fmm p=8 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=8, fast_multipole_theta=0.5)),
    ("fmm p=6 theta=0.5 tensor", dict(coulomb_method="fast-multipole", fast_multipole_order=6, fast_multipole_theta=0.5,
                                      precision="tensor")),
    ("fmm p=7 theta=0.5 tensor", dict(coulomb_method="fast-multipole", fast_multipole_order=7, fast_multipole_theta=0.5,
                                      precision="tensor")),
    ("learned p=2 + MLP theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=2,
                                        fast_multipole_theta=0.5, fmm_learned=1, learned_audit_interval=0)),
]
PLAIN_P6 = "fmm p=6 theta=0.5"
# training of the learned correction: particles of 8,192 sampled leaves,
# 8,000 Adam steps of 4,096 samples (outside the timed region)
LEARNED_TRAINING = dict(sample_leaves=8192, steps=8000, batch=4096, lr=5e-4)
LEARNED = "learned p=2 + MLP theta=0.5"

# DRAM traffic (read + write) per launch of the FMM's M2L class-product kernel,
# by order, from ncu captures of one launch (launches at N = 1,048,576 process
# chunks of the same bounded size).
# DRAM traffic per class pair of the tensor-core product kernel (the FP32
# per-pair products written, the split expansions read past L2), from one
# ncu launch at 262,144 particles scaled by the pairs of a launch here.
TC_PRODUCT_TRAFFIC_PER_PAIR = {
    7: (519.0, "ncu dram__bytes_read.sum + dram__bytes_write.sum of m2l_class_tc_kernel<7> on 262,144 particles "
               "(leaf 128, 2,973,968 class pairs: 0.152 GB read + 1.393 GB written = 519 B per pair), scaled by "
               "this launch's class pairs; profiles/m2l_class_tc_kernel_tree262k_leaf128.md"),
}
NEAR_TRAFFIC_PER_PAIR = (
    0.0300, "ncu dram__bytes_read.sum + dram__bytes_write.sum of fmm_p2p32_kernel on 262,144 particles (leaf 128, "
            "1.374 G particle pairs: 12.9 MB read + 28.4 MB written = 0.030 B per pair), scaled by this launch's "
            "pairs; profiles/fmm_p2p32_kernel_tree262k_leaf128.md")
FMM_PRODUCT_TRAFFIC = {
    7: (5.18e9, "ncu dram__bytes_read.sum + dram__bytes_write.sum of m2l_class_mma_kernel<7>, mean of two launches "
                "of 4.47 M pairs each (0.89 / 1.10 GB read + 4.18 GB written: the per-pair products), "
                "profiles/m2l_class_mma_kernel_tree1m.md"),
    8: (5.17e9, "ncu dram__bytes_read.sum + dram__bytes_write.sum of m2l_class_mma_kernel<8>, mean of two launches "
                "of 3.25 M pairs each (0.92 GB read + 4.26 GB written: the per-pair products), "
                "profiles/m2l_class_mma_kernel_tree1m.md"),
}


def tree_cloud(n=1 << 20, seed=42):
    """N positrons, Gaussian cloud sigma 1e-4, 1e-4, 3e-4 m, 5 K Maxwellian."""
    rng = np.random.default_rng(seed)
    pos = rng.normal(0.0, 1.0, (n, 3)) * np.array([1e-4, 1e-4, 3e-4])
    vel = rng.normal(0.0, 1.0, (n, 3)) * np.sqrt(KB * 5.0 / MASS[1])
    return pos, vel, np.ones(n, np.uint8)


def tree_config(n, world):
    """The workload description; both arms print exactly this dict."""
    return {"workload": (f"tree solvers on N={n:,} positrons: Gaussian cloud sigma 1e-4 x 1e-4 x 3e-4 m, "
                         "5 K Maxwellian, b0=1 T, U=10 V, z0=rho0=0.01 m, dt=8.931e-12 s, cooling and "
                         "annihilation off; one step = Coulomb force + Boris push of the whole cloud"),
            "n_particles": n, "seed": 42,
            "methods": [name for name, _ in TREE_METHODS],
            "selection": "value = fastest method whose RMS relative force error vs the FP64 exact sum "
                         "is <= 1e-5 (4,096 evenly spaced audited particles); the table also holds the FMM "
                         "order/theta/leaf the library's autotuner picks under that budget",
            "error_budget": ERROR_BUDGET,
            "l2": "flushed between timed steps by a 256 MiB write (outside the per-step events)",
            "parallelism": f"replicas x{world} (a single instance does not shard)"}


def tree_params(n, over):
    import amk
    kw = dict(seed=42, b0=1.0, trap_voltage=10.0, z0=0.01, rho0=0.01, num_steps=500,
              populations={"positron": n}, temperatures={"positron": 5.0}, cloud_radii=(1e-4, 1e-4, 3e-4),
              bath_temperature=0.0, cooling_scale=0.0, cooling_enabled=0, coulomb_forces_enabled=1,
              energy_method="allpairs", annihilation_enabled=0)
    kw.update(over)
    return amk.make_params(**kw)


def cpu_tree_step(x, y, z, vx, vy, vz, order=6, theta=0.5):
    """One reference CPU step on the sample: the reference's own FMM
    (fast-multipole.cc via oracle/_ref, OpenMP on all host cores) for the
    Coulomb force, then the FP64 Boris push of the sample. Returns seconds."""
    O = _oracle()
    n = len(x)
    q = np.full(n, E)
    m = np.full(n, MASS[1])
    t0 = time.perf_counter()
    (fx, fy, fz), _ = O.ref_fmm(x, y, z, q, order, theta)
    state = dict(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, q=q, m=m, alive=np.ones(n, np.uint8))
    O.boris_push(state, fx, fy, fz, 1.0, 10.0, 0.01, 0.01, 8.930966882e-12, False)
    return time.perf_counter() - t0


def cpu_tree_baseline(pos, vel, n_sample, warm, steps):
    O = _oracle()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libamkref.so is missing: build it with `make -C oracle ref`")
    x, y, z = (np.ascontiguousarray(pos[:n_sample, k]) for k in range(3))
    vx, vy, vz = (np.ascontiguousarray(vel[:n_sample, k]) for k in range(3))
    times = []
    for k in range(warm + steps):
        t = cpu_tree_step(x, y, z, vx, vy, vz)
        if k >= warm:
            times.append(t)
    total = float(sum(times))
    return {"value": n_sample * steps / total, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "sample": (f"first {n_sample:,} particles of the same cloud; per step the reference's own FMM "
                       f"(fast-multipole.cc, p=6, theta=0.5, leaf 32, OpenMP on all host cores) + FP64 Boris "
                       f"push of the sample; {steps} timed steps after {warm} untimed; the reference FMM's "
                       "cost per particle at this size is within 15% of its cost at 1,048,576 particles"),
            "ms_per_step": 1e3 * total / steps}


def run_reference_tree(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    pos, vel, _ = tree_cloud(args.tree_n)
    n_s = min(args.ref_sample, len(pos))
    cpu = cpu_tree_baseline(pos, vel, n_s, args.warmup, args.steps)
    line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian cloud, numpy default_rng(42))",
            "config": tree_config(len(pos), world),
            "cpu_baseline": {k: v for k, v in cpu.items() if k != "ms_per_step"},
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def tree_method_entry(sim, name, over, args, stream, flusher):
    """Audit and time one method on a fresh context holding the cloud."""
    entry = {}
    if over.get("fmm_learned"):
        t0 = time.perf_counter()
        loss, samples = sim.fmm_train_correction(0.5, **LEARNED_TRAINING)
        entry["training"] = {"seconds": round(time.perf_counter() - t0, 2), "samples": samples,
                             "final_loss": loss}
    sim.coulomb()
    rms, mx = sim.force_error(args.audit_samples)
    entry.update({"rms_rel": rms, "max_rel": mx, "meets_1e-5": bool(rms <= ERROR_BUDGET)})
    sim.step(2)
    sim.synchronize()
    k = max(1, min(args.steps, args.method_steps))
    ms = timed_steps(sim, stream, flusher, k) / k
    entry.update(ms_per_step=ms, value=sim.num_particles() / (ms * 1e-3), steps=k)
    sim.set_profiling(True)
    sim.reset_phase_times()
    sim.step(1)
    sim.synchronize()
    entry["phase_ms"] = {kk: round(v[0], 3) for kk, v in sim.phase_times().items() if v[1]}
    sim.set_profiling(False)
    return entry


def measured_peak(key, fallback):
    """A figure of the pool's measured-peaks file (MEASURED_PEAKS.json beside
    this script) and where it came from, else the stated fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            v = json.load(fh).get(key)
        if isinstance(v, (int, float)) and v > 0:
            return float(v), f"of measured ({key} in MEASURED_PEAKS.json)"
    except (OSError, ValueError):
        pass
    return fallback, f"of fallback ({fallback:g}; no {key} in a MEASURED_PEAKS.json)"


def tree_roofline(sim, over, n):
    if over["coulomb_method"] == "allpairs":
        sim.set_profiling(True)
        sim.reset_phase_times()
        sim.step(1)
        sim.synchronize()
        ap_ms, ap_n = sim.phase_times()["allpairs"]
        sim.set_profiling(False)
        peak = sim.measure_fp32_peak()
        achieved = 20.0 * n * (n - 1) / (ap_ms / ap_n * 1e-3) / 1e12
        return {"bound": "fp32", "kernel": "allpairs_kernel", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": 3.276e6 * n / 65536,
                "traffic_source": "ncu capture at N = 65,536 (profiles/allpairs_kernel_direct65k.md), scaled by N",
                "peak_source": "measured in this run: FFMA probe kernel over all SMs (2 flop/FFMA)",
                "flop_convention": "20 flop per pair interaction x N(N-1) pairs",
                "avg_launch_ms": ap_ms / ap_n}
    if over["coulomb_method"] == "fast-multipole" and not over.get("fmm_learned"):
        sim.set_profiling(True)
        sim.reset_phase_times()
        sim.step(1)
        sim.synchronize()
        ph = sim.phase_times()
        sim.set_profiling(False)
        prod_ms, prod_n = ph["fmm_m2l_products"]
        st = sim.fmm_stats()
        p_ = st["order"]
        nm = (p_ + 1) * (p_ + 2) * (p_ + 3) // 6
        achieved = 2.0 * nm * nm * st["m2l_class_pairs"] / (prod_ms * 1e-3) / 1e12
        if over.get("precision") == "tensor" and 5 <= p_ <= 7:
            bf16, src = measured_peak("bf16_tflops", 1590.0)
            per_pair = TC_PRODUCT_TRAFFIC_PER_PAIR.get(p_)
            traffic = None if per_pair is None else per_pair[0] * st["m2l_class_pairs"] / max(1, prod_n)
            products = {"bound": "tensor (split BF16)", "kernel": f"m2l_class_tc_kernel<{p_}>", "achieved": achieved,
                        "peak": bf16 / 6.0, "unit": "TFLOP/s", "frac": achieved / (bf16 / 6.0), "traffic": traffic,
                        "traffic_source": None if per_pair is None else per_pair[1],
                        "peak_source": f"dense BF16 tensor peak {src}, divided by the six BF16 products each "
                                       "split-BF16 product issues",
                        "flop_convention": f"2 n_m^2 flop (n_m = {nm}) per M2L pair evaluated as a class product "
                                           f"({st['m2l_class_pairs']:,} of {st['m2l_pairs']:,} pairs)",
                        "avg_launch_ms": prod_ms / max(1, prod_n), "launches_per_step": prod_n,
                        "m2l_phase_ms": ph["fmm_m2l"][0], "classes": st["m2l_classes"]}
            near_ms, near_n = ph.get("fmm_near", (0.0, 0))
            if not near_n:
                return products
            pairs = st["p2p_particle_pairs"]
            near_avg = near_ms / near_n
            peak32 = sim.measure_fp32_peak()
            ach32 = 20.0 * pairs / (near_avg * 1e-3) / 1e12
            near = {"bound": "fp32", "kernel": "fmm_p2p32_kernel", "achieved": ach32, "peak": peak32,
                    "unit": "TFLOP/s", "frac": ach32 / peak32,
                    "traffic": NEAR_TRAFFIC_PER_PAIR[0] * pairs, "traffic_source": NEAR_TRAFFIC_PER_PAIR[1],
                    "peak_source": "measured in this run: FFMA probe kernel over all SMs (2 flop/FFMA)",
                    "flop_convention": f"20 flop per particle pair of the P2P leaf pairs ({pairs:,} pairs, the "
                                       "particle itself included), as for the all-pairs kernel",
                    "avg_launch_ms": near_avg, "launches_per_step": near_n,
                    "timing": "CUDA events on the near-field stream, which it shares with nothing; the kernel "
                              "runs concurrently with the per-pair M2L products, the per-target M2L sums and L2L"}
            dominant, other = (near, products) if near_avg >= products["avg_launch_ms"] else (products, near)
            dominant["other_kernel"] = other
            return dominant
        peak = sim.measure_fp64_peak()
        traffic = FMM_PRODUCT_TRAFFIC.get(p_)
        return {"bound": "fp64 tensor", "kernel": f"m2l_class_mma_kernel<{p_}>", "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None if traffic is None else traffic[0],
                "traffic_source": None if traffic is None else traffic[1],
                "peak_source": "measured in this run: mma.m8n8k4 FP64 probe kernel over all SMs "
                               "(512 flop per warp instruction); the driver's peak file has no FP64 figure",
                "flop_convention": f"2 n_m^2 flop (n_m = {nm}) per M2L pair evaluated as a class product "
                                   f"({st['m2l_class_pairs']:,} of {st['m2l_pairs']:,} pairs; the rest take "
                                   "the per-pair path)",
                "avg_launch_ms": prod_ms / max(1, prod_n), "launches_per_step": prod_n,
                "m2l_phase_ms": ph["fmm_m2l"][0], "classes": st["m2l_classes"]}
    return None


def run_tree(args):
    import torch
    import amk
    world, rank, local = dist_setup()
    init_nccl(world, local)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    pos, vel, sp = tree_cloud(args.tree_n)
    n = len(pos)
    methods = [m for m in TREE_METHODS if not args.tree_methods or m[0] in args.tree_methods.split(",")]
    if not methods:
        raise SystemExit(f"--tree-methods: none of {[m[0] for m in TREE_METHODS]}")

    overs = dict(TREE_METHODS)

    def new_sim(over):
        sim = amk.Simulation(tree_params(n, {k: v for k, v in over.items() if k not in ("leaf", "precision")}),
                             device=local)
        if "leaf" in over:
            sim.set_leaf_sizes(fmm_leaf=over["leaf"])
        elif args.fmm_leaf and over.get("coulomb_method") == "fast-multipole":
            sim.set_leaf_sizes(fmm_leaf=args.fmm_leaf)
        if "precision" in over:
            sim.set_fmm_precision(over["precision"])
        sim.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], sp)
        stream = torch.cuda.ExternalStream(sim.stream(), device=device)
        return sim, stream

    results, best = {}, None
    for name, over in methods:
        sim, stream = new_sim(over)
        entry = tree_method_entry(sim, name, over, args, stream, Flusher(device, stream))
        results[name] = entry
        if entry["meets_1e-5"] and (best is None or entry["value"] > results[best]["value"]):
            best = name
        sim.close()
    if args.autotune:
        # the FMM configuration (order 4..8, theta 0.5..0.4, leaf 16..256;
        # tensor-core M2L products for orders 5-7) the library's autotuner
        # finds fastest within the budget
        sim, stream = new_sim(dict(overs[PLAIN_P6], precision="tensor"))
        t0 = time.perf_counter()
        try:
            cands, ch = sim.autotune(ERROR_BUDGET, samples=args.audit_samples, flags=1 | 4)  # FMM only
        except amk.AmkError:
            cands, ch = [], -1
        tune_s = time.perf_counter() - t0
        sim.close()
        if ch >= 0:
            w = cands[ch]
            name = f"fmm autotuned p={w['order']} theta={w['theta']} leaf={w['leaf']}"
            name += " tensor" if 5 <= w["order"] <= 7 else ""
            overs[name] = dict(coulomb_method="fast-multipole", fast_multipole_order=w["order"],
                               fast_multipole_theta=w["theta"], leaf=w["leaf"], precision="tensor")
            sim, stream = new_sim(overs[name])
            entry = tree_method_entry(sim, name, overs[name], args, stream, Flusher(device, stream))
            sim.close()
            entry["autotune"] = {"seconds": round(tune_s, 1), "candidates": [
                [c["order"], c["theta"], c["leaf"], round(c["ms"], 2), c["rms"]] for c in cands if c["ms"] > 0],
                "columns": ["order", "theta", "leaf", "ms per force call", "rms"]}
            results[name] = entry
            if entry["meets_1e-5"] and (best is None or entry["value"] > results[best]["value"]):
                best = name

    # ---- the chosen method: W untimed steps, exactly K timed steps
    name = best if best is not None else methods[0][0]
    over = overs[name]
    sim, stream = new_sim(over)
    flusher = Flusher(device, stream)
    if over.get("fmm_learned"):
        sim.fmm_train_correction(0.5, **LEARNED_TRAINING)
    for _ in range(args.warmup):
        sim.step(1)
        flusher()
    sim.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = sim.kernel_launches()
    total_ms = timed_steps(sim, stream, flusher, args.steps)
    if world > 1:
        torch.distributed.barrier()
    launches = sim.kernel_launches() - launches0
    clocks = sampler.stop()
    total_ms = max_over_ranks(total_ms, world, device)
    value = world * n * args.steps / (total_ms * 1e-3)
    roofline = tree_roofline(sim, over, n)
    e2e_ms, h2d, d2h = e2e_through_abi(sim, stream, n, args.steps)
    e2e_ms = max_over_ranks(e2e_ms, world, device)
    e2e = {"value": world * n * args.steps / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "steps": args.steps,
           "api": "amk_update_state + amk_step + amk_get_particles (pinned host buffers)"}
    sim.close()

    learned_vs_p6 = None
    if LEARNED in results and PLAIN_P6 in results:
        a, b = results[LEARNED], results[PLAIN_P6]
        learned_vs_p6 = {"ratio": a["value"] / b["value"], "learned_rms": a["rms_rel"], "p6_rms": b["rms_rel"],
                         "both_within_budget": bool(a["meets_1e-5"] and b["meets_1e-5"]),
                         "target": ">= 3x at <= 1e-5 RMS"}

    sweep = None
    if args.sweep_ratio and world == 1:
        sweep = measure_sweep(args, 1, 0, local, device, ratio_only=True)

    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline:
        cpu = cpu_tree_baseline(pos, vel, min(args.ref_sample, n), 1, 3)
        cpu.pop("ms_per_step")
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": ("fp32" if over["coulomb_method"] == "allpairs" else
                          "bf16x3 M2L products, f32 near field, f64 expansions and push"
                          if over.get("precision") == "tensor" else "f64"),
                "data": "synthetic (seeded Gaussian cloud, numpy default_rng(42))",
                "config": tree_config(n, world), "chosen": name, "methods": results,
                "learned_vs_plain_p6": learned_vs_p6, "sweep_batched_vs_one_at_a_time": sweep,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    finish_dist(world)
    return 0


# ================================================================== direct65k
DIRECT_POPS = {"antiproton": 32768, "positron": 32768}


def direct_config(world):
    return {"workload": "direct all-pairs Coulomb + Boris push, N=65,536 (32,768 e+ + 32,768 pbar), uniform "
                        "ellipsoid 2e-4 x 2e-4 x 5e-4 m, 10 K Maxwellian, b0=3 T, U=50 V, z0=rho0=0.01 m, "
                        "dt=2.977e-12 s",
            "n_particles": 65536, "seed": 42, "cooling": False, "annihilation": False,
            "state_precision": "fp64 positions/velocities",
            "l2": "flushed between steps by a 256 MiB write (inputs 6.5 MB < L2)",
            "parallelism": f"replicas x{world} (a single instance does not shard)"}


def direct_params():
    import amk
    return amk.make_params(
        seed=42, b0=3.0, trap_voltage=50.0, z0=0.01, rho0=0.01, num_steps=1000,
        populations=dict(DIRECT_POPS), temperatures={"antiproton": 10.0, "positron": 10.0},
        cloud_radii=(2e-4, 2e-4, 5e-4), bath_temperature=0.0, cooling_scale=0.0,
        cooling_enabled=0, coulomb_forces_enabled=1, coulomb_method="allpairs",
        energy_method="allpairs", annihilation_enabled=0)


def cpu_direct_step_time(x, y, z, q, m, n_sample, seed=0):
    """Reference CPU step on a bounded sample: the reference's Barnes-Hut tree
    at theta = 0 (exact all-pairs) over all N sources walked for n_sample
    targets, plus the FP64 push of those targets. Returns (seconds,
    targets, forces)."""
    O = _oracle()
    n = len(x)
    rng = np.random.default_rng(seed)
    targets = np.sort(rng.choice(n, n_sample, replace=False))
    t0 = time.perf_counter()
    f = O.ref_bh_forces_subset(x, y, z, q, 0.0, targets, 8)
    state = dict(x=x[targets].copy(), y=y[targets].copy(), z=z[targets].copy(), vx=np.zeros(n_sample),
                 vy=np.zeros(n_sample), vz=np.zeros(n_sample), q=q[targets], m=m[targets],
                 alive=np.ones(n_sample, np.uint8))
    O.boris_push(state, f[0], f[1], f[2], 3.0, 50.0, 0.01, 0.01, 2.977e-12, False)
    return time.perf_counter() - t0, targets, f


def direct_cloud():
    O = _oracle()
    pos = O.initial_positions(DIRECT_POPS, [2e-4, 2e-4, 5e-4], 42)
    sp = O.species_column(DIRECT_POPS)
    m, q = O.species_props(sp)
    return pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), q, m


def run_reference_direct(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    x, y, z, q, m = direct_cloud()
    times = []
    for k in range(args.warmup + args.steps):
        t, _, _ = cpu_direct_step_time(x, y, z, q, m, args.ref_sample_direct, seed=k)
        if k >= args.warmup:
            times.append(t)
    total = float(sum(times))
    value = args.ref_sample_direct * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference initial-condition generator, seed 42)", "config": direct_config(world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"per step: the reference's exact (theta=0) Barnes-Hut tree over all "
                                       f"65,536 sources walked for {args.ref_sample_direct} random targets + FP64 "
                                       "push of those targets; value counts the targets processed"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_direct(args):
    import torch
    import amk
    world, rank, local = dist_setup()
    init_nccl(world, local)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    sim = amk.Simulation(direct_params(), device=local)
    sim.init_particles()
    n = sim.num_particles()
    stream = torch.cuda.ExternalStream(sim.stream(), device=device)
    flusher = Flusher(device, stream)
    for _ in range(args.warmup):
        sim.step(1)
        flusher()
    sim.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = sim.kernel_launches()
    total_ms = timed_steps(sim, stream, flusher, args.steps)
    if world > 1:
        torch.distributed.barrier()
    launches = sim.kernel_launches() - launches0
    clocks = sampler.stop()
    total_ms = max_over_ranks(total_ms, world, device)
    value = world * n * args.steps / (total_ms * 1e-3)

    prof_steps = min(args.steps, 50)
    sim.set_profiling(True)
    sim.reset_phase_times()
    for _ in range(prof_steps):
        sim.step(1)
        flusher()
    sim.synchronize()
    phases = sim.phase_times()
    sim.set_profiling(False)
    ap_ms, ap_launches = phases["allpairs"]
    ap_avg_ms = ap_ms / max(ap_launches, 1)
    flops_per_launch = 20.0 * n * (n - 1)
    achieved = flops_per_launch / (ap_avg_ms * 1e-3) / 1e12
    peak = sim.measure_fp32_peak()
    roofline = {"bound": "fp32", "kernel": "allpairs_kernel", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": 3.276e6,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one allpairs_kernel "
                                  "launch of this workload (profiles/allpairs_kernel_direct65k.md)",
                "peak_source": "measured in this run: FFMA probe kernel over all SMs "
                               "(2 flop/FFMA); no FP32 figure in the driver's peak file",
                "flops_per_launch": flops_per_launch,
                "flop_convention": "20 flop per pair interaction x N(N-1) pairs",
                "avg_launch_ms": ap_avg_ms,
                "phase_ms_per_step": {k: v[0] / max(prof_steps, 1) for k, v in phases.items() if v[1]}}
    e2e_ms, h2d, d2h = e2e_through_abi(sim, stream, n, args.steps)
    e2e_ms = max_over_ranks(e2e_ms, world, device)
    e2e = {"value": world * n * args.steps / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "steps": args.steps,
           "api": "amk_update_state + amk_step + amk_get_particles (pinned host buffers)"}
    cpu = err = None
    if rank == 0 and world == 1 and args.cpu_baseline:
        st = sim.get_particles()
        sim.coulomb_allpairs()
        fx, fy, fz = sim.get_forces()
        _, _, _, q, m = direct_cloud()
        t, targets, fref = cpu_direct_step_time(st["x"], st["y"], st["z"], q, m, args.cpu_sample)
        cpu = {"value": args.cpu_sample / t, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
               "sample": f"the reference's exact (theta=0) Barnes-Hut tree over all {n} sources walked for "
                         f"{args.cpu_sample} random targets + FP64 push of those targets; OpenMP on all host "
                         "cores; value counts the targets processed"}
        num = np.sqrt((fx[targets] - fref[0]) ** 2 + (fy[targets] - fref[1]) ** 2 + (fz[targets] - fref[2]) ** 2)
        den = np.sqrt(fref[0] ** 2 + fref[1] ** 2 + fref[2] ** 2)
        rel = num / den
        err = {"rms_rel": float(np.sqrt(np.mean(rel ** 2))), "max_rel": float(np.max(rel)),
               "targets": int(len(targets)), "against": "the reference's FP64 exact sum"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic (reference initial-condition generator, seed 42)",
                "config": direct_config(world), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clocks, "force_error_vs_fp64": err}
        print(json.dumps(line), flush=True)
    sim.close()
    finish_dist(world)
    return 0


# ================================================================== sweep512
def make_sweep(n_inst=512, seed=2024, method_split=8192, order=4):
    """The batched sweep: n_inst independent trap instances, populations
    log-uniform in [1e2, 1e5] (even, 1:1 species pairs e-/e+ or e+/pbar per
    instance), temperatures log-uniform 4..1e4 K, b0 U(1, 5) T, trap_voltage
    U(5, 50) V, cloud radii U(5e-5, 5e-4) m per axis (uniform ellipsoid),
    Maxwellian velocities, cooling (bath 4 K, scale 1) and annihilation
    (contact 5e-6 m, p = 0.5) on. Coulomb: all-pairs below `method_split`
    particles, FMM of `order` (theta 0.5) from there (method_split=None: all
    instances all-pairs). Returns [(pos, vel, species, params)]."""
    import amk
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_inst):
        n = max(2, int(round(10 ** rng.uniform(2.0, 5.0))) // 2 * 2)
        pair = (3, 1) if rng.random() < 0.5 else (1, 0)  # (electron, positron) / (positron, antiproton)
        temp = 10 ** rng.uniform(np.log10(4.0), 4.0)
        b0 = rng.uniform(1.0, 5.0)
        volt = rng.uniform(5.0, 50.0)
        radii = rng.uniform(5e-5, 5e-4, 3)
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        pos = d * rng.random((n, 1)) ** (1.0 / 3.0) * radii
        sp = np.repeat(np.array(pair, np.uint8), n // 2)
        m = np.array([MASS[int(k)] for k in pair]).repeat(n // 2)
        vel = rng.normal(size=(n, 3)) * np.sqrt(KB * temp / m)[:, None]
        names = {0: "antiproton", 1: "positron", 3: "electron"}
        method = "allpairs" if method_split is None or n < method_split else "fast-multipole"
        p = amk.make_params(seed=1000 + i, b0=b0, trap_voltage=volt, z0=0.01, rho0=0.01,
                            populations={names[pair[0]]: n // 2, names[pair[1]]: n // 2},
                            temperatures={names[pair[0]]: temp, names[pair[1]]: temp},
                            cloud_radii=tuple(radii), bath_temperature=4.0, cooling_scale=1.0,
                            cooling_enabled=1, coulomb_forces_enabled=1, coulomb_method=method,
                            energy_method="allpairs", cutoff_radius=1e-5, fast_multipole_order=order,
                            fast_multipole_theta=0.5, annihilation_enabled=1, contact_radius=5e-6,
                            annihilation_probability=0.5)
        out.append((pos, vel, sp, p))
    return out


def load_sweep(sim, insts):
    pos = np.concatenate([i[0] for i in insts])
    vel = np.concatenate([i[1] for i in insts])
    sp = np.concatenate([i[2] for i in insts])
    sim.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], sp)
    offsets = np.concatenate([[0], np.cumsum([len(i[0]) for i in insts])])
    sim.batch_set([i[3] for i in insts], offsets)
    return pos, vel, sp, offsets


def sweep_share(insts, world, rank):
    """This rank's instances of the sweep (LPT on the per-instance cost model)."""
    from amk import partition
    costs = [partition.instance_cost(len(i[0]), int(i[3].coulomb_method)) for i in insts]
    parts = partition.partition_lpt(costs, world)
    return parts[rank], partition.imbalance(costs, parts)


def measure_sweep(args, world, rank, local, device, ratio_only=False):
    """Batched sweep (one persistent all-pairs launch, CUDA-graph chunks) on
    this rank's share of the instances, against the same instances stepped one
    at a time with the single-instance kernels. Returns a dict of results."""
    import torch
    import amk
    all_insts = make_sweep(n_inst=args.instances, seed=2024, method_split=None)
    mine, imb = sweep_share(all_insts, world, rank)
    insts = [all_insts[i] for i in mine]
    n_total = int(sum(len(i[0]) for i in insts))
    sim = amk.Simulation(device=local)
    load_sweep(sim, insts)
    t0 = time.perf_counter()
    methods = sim.batch_autotune(error_budget=ERROR_BUDGET, samples=256)
    tune_s = time.perf_counter() - t0
    names = {-1: "none", 0: "cutoff", 1: "barnes-hut", 2: "fmm", 3: "allpairs"}
    method_counts = {names[int(m)]: int((methods == m).sum()) for m in np.unique(methods)}
    steps = args.sweep_steps if ratio_only else args.steps
    chunk = min(100, steps)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def live():
        return int(sim.batch_status()["alive"].sum())

    def timed(fn):
        st = torch.cuda.ExternalStream(sim.stream(), device=device)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        ev0.record(st)
        fn()
        ev1.record(st)
        torch.cuda.synchronize()
        barrier()
        return ev0.elapsed_time(ev1)

    def live_sum(v):  # live particles summed over ranks
        if world == 1:
            return float(v)
        t = torch.tensor([float(v)], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t)
        return float(t.item())

    # warm-up: plain steps (the first is the staggered one), then one chunk to
    # capture and instantiate the graph outside the timed region
    sim.batch_step(args.warmup)
    sim.batch_step(chunk, graph_chunk=chunk)
    sim.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = sim.kernel_launches()
    live0 = live_sum(live())
    ms = timed(lambda: sim.batch_step(steps, graph_chunk=chunk))
    live1 = live_sum(live())
    launches = sim.kernel_launches() - launches0
    clocks = sampler.stop()
    ms = max_over_ranks(ms, world, device)
    value = 0.5 * (live0 + live1) * steps / (ms * 1e-3)

    serial_steps = max(1, min(steps, args.serial_steps))
    sim.batch_step(1, serial=True)  # untimed: grows the single-instance scratch to its largest size
    s_live0 = live_sum(live())
    serial_ms = max_over_ranks(timed(lambda: sim.batch_step(serial_steps, serial=True)), world, device)
    serial_value = 0.5 * (s_live0 + live_sum(live())) * serial_steps / (serial_ms * 1e-3)
    out = {"batched_value": value, "one_at_a_time_value": serial_value, "ratio": value / serial_value,
           "target": ">= 5x", "instances": len(insts), "particles": n_total, "steps": steps,
           "one_at_a_time_steps": serial_steps, "graph_chunk": chunk,
           "autotune": {"methods": method_counts, "seconds": round(tune_s, 2)},
           "rate_counts": "live (not yet annihilated) particles, mean of the timed window's start and end"}
    if ratio_only:
        sim.close()
        return out

    prof_steps = 2
    sim.set_profiling(True)
    sim.reset_phase_times()
    sim.batch_step(prof_steps)
    sim.synchronize()
    phases = sim.phase_times()
    sim.set_profiling(False)
    ap_ms, ap_launches = phases["allpairs"]
    ap_avg = ap_ms / max(ap_launches, 1)
    alive_i = sim.batch_status()["alive"].astype(np.float64)
    pairs = float(sum(a * (a - 1) for a, m in zip(alive_i, methods) if m == 3))
    peak = sim.measure_fp32_peak()
    achieved = 20.0 * pairs / (ap_avg * 1e-3) / 1e12
    out["roofline"] = {
        "bound": "fp32", "kernel": "batch_allpairs_kernel", "achieved": achieved, "peak": peak,
        "unit": "TFLOP/s", "frac": achieved / peak, "traffic": 116.2e6 * n_total / 1380664,
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of batch_allpairs_kernel on the "
                          "64-instance case (116.2 MB for 1,380,664 particles, "
                          "profiles/batch_allpairs_kernel_sweep.md), scaled by particle count",
        "peak_source": "measured in this run: FFMA probe kernel over all SMs (2 flop/FFMA)",
        "flops_per_launch": 20.0 * pairs,
        "flop_convention": "20 flop per pair interaction x sum_i A_i(A_i-1), A_i the live particles of "
                           "all-pairs instance i",
        "avg_launch_ms": ap_avg,
        "phase_ms_per_step": {k: v[0] / prof_steps for k, v in phases.items() if v[1]}}

    e2e_steps = max(1, min(steps, 10))
    sim.close()
    sim = amk.Simulation(device=local)
    load_sweep(sim, insts)
    sim.batch_step(args.warmup)
    st = torch.cuda.ExternalStream(sim.stream(), device=device)
    e_live0 = live_sum(live())
    barrier()
    e2e_ms, h2d, d2h = e2e_through_abi(sim, st, n_total, e2e_steps, step_fn=lambda: sim.batch_step(1))
    e2e_ms = max_over_ranks(e2e_ms, world, device)
    out["e2e"] = {"value": 0.5 * (e_live0 + live_sum(live())) * e2e_steps / (e2e_ms * 1e-3), "unit": UNIT,
                  "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                  "api": "amk_update_state + amk_batch_step + amk_get_particles (pinned host buffers)"}
    # one host gather of per-instance results (live count, total energy) in instance order
    from amk import partition
    status = sim.batch_status()
    energies = sim.batch_energy()
    rows = [(int(a), float(e["total"])) for a, e in zip(status["alive"], energies)]
    gathered = partition.gather_instance_rows(mine, rows, len(all_insts), world, rank)
    out["per_instance"] = None if gathered is None else {
        "instances": len(gathered), "alive_total": int(sum(r[0] for r in gathered))}
    out.update(value=value, ms=ms, launches=launches, clocks=clocks, imbalance=imb,
               contact_overflow=bool(status["overflow"]), insts=insts, n_total=n_total)
    sim.close()
    return out


def cpu_sweep_baseline(insts, pair_budget):
    """The reference's CPU code on a bounded sample of the sweep: instances in
    index order (a random sample: instance parameters are drawn independently)
    until their N_i^2 pair counts reach `pair_budget`; each instance the
    reference's exact (theta=0) Barnes-Hut tree over all its sources walked
    for all its particles, plus the FP64 push. Returns (instances, particles
    processed, seconds)."""
    O = _oracle()
    total, parts, pairs, k = 0.0, 0, 0.0, 0
    for pos, vel, sp, p in insts:
        n = len(pos)
        if k > 0 and pairs + float(n) * n > pair_budget:
            continue
        m, q = O.species_props(sp)
        x, y, z = pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()
        t0 = time.perf_counter()
        f = O.ref_bh_forces(x, y, z, q, 0.0, 8)
        state = dict(x=x, y=y, z=z, vx=vel[:, 0].copy(), vy=vel[:, 1].copy(), vz=vel[:, 2].copy(),
                     q=q, m=m, alive=np.ones(n, np.uint8))
        O.boris_push(state, f[0], f[1], f[2], p.b0, p.trap_voltage, p.z0, p.rho0, p.dt, False)
        total += time.perf_counter() - t0
        parts += n
        pairs += float(n) * n
        k += 1
    return k, parts, total


def sweep_config(args, world):
    return {"workload": f"batched sweep: {args.instances} trap instances, N_i log-uniform 1e2..1e5, e-/e+ or "
                        "e+/pbar 1:1, T 4..1e4 K, b0 1..5 T, U 5..50 V, radii 5e-5..5e-4 m, cooling (4 K) and "
                        "annihilation (5e-6 m, p=0.5) on",
            "instances": args.instances, "seed": 2024,
            "solver": "per-instance method chosen by amk_batch_autotune under a 1e-5 RMS force-error budget; "
                      "all-pairs instances share one persistent launch (cost-ordered work queue); FP64 state",
            "l2": "not flushed: state of about 8 M particles (> 700 MB) exceeds L2",
            "parallelism": f"dp{world}: the instances partitioned across ranks (LPT on a per-instance cost "
                           "model), no per-step collective, one host gather at the end"}


def run_sweep(args):
    import torch
    world, rank, local = dist_setup()
    init_nccl(world, local)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    r = measure_sweep(args, world, rank, local, device)
    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline:
        k, parts, secs = cpu_sweep_baseline(r["insts"], args.ref_pairs)
        cpu = {"value": parts / secs, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
               "sample": f"{k} instances of this rank's share in index order, up to {args.ref_pairs:.0e} "
                         "particle pairs (instances that would exceed it are skipped): per instance the reference's exact (theta=0) Barnes-Hut tree walked "
                         "for all its particles + FP64 push; value counts the particles processed"}
    if rank == 0:
        sizes = np.array([len(i[0]) for i in r["insts"]])
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic (seeded sweep generator)", "config": sweep_config(args, world),
                "rank0_share": {"instances": r["instances"], "particles": r["particles"],
                                "sizes": {"min": int(sizes.min()), "median": int(np.median(sizes)),
                                          "max": int(sizes.max())},
                                "load_imbalance": r["imbalance"]},
                "roofline": r["roofline"], "cpu_baseline": cpu, "e2e": r["e2e"], "gpu_launches": r["launches"],
                "clocks": r["clocks"],
                "one_at_a_time": {"value": r["one_at_a_time_value"], "steps": r["one_at_a_time_steps"],
                                  "speedup_batched": r["ratio"]},
                "autotune": r["autotune"], "per_instance_gather": r["per_instance"],
                "contact_overflow": r["contact_overflow"]}
        print(json.dumps(line), flush=True)
    finish_dist(world)
    return 0


def run_reference_sweep(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    insts = sweep_instances_numpy(args.instances)
    times, parts, k_inst = [], 0, 0
    for k in range(args.warmup + args.steps):
        k_inst, p, t = cpu_sweep_baseline(insts, args.ref_pairs)
        if k >= args.warmup:
            times.append(t)
            parts = p
    total = float(sum(times))
    value = parts * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded sweep generator)", "config": sweep_config(args, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"per step {k_inst} instances in index order, up to {args.ref_pairs:.0e} "
                                       "particle pairs (instances that would exceed it are skipped): the reference's exact (theta=0) Barnes-Hut tree walked "
                                       "for all their particles + FP64 push; value counts the particles processed"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


class _SweepParams:
    """The few per-instance parameters the CPU sweep leg reads."""

    def __init__(self, b0, volt, species):
        O = _oracle()
        self.b0, self.trap_voltage, self.z0, self.rho0 = b0, volt, 0.01, 0.01
        self.dt = O.dt_for(list(species), b0)


def sweep_instances_numpy(n_inst, seed=2024):
    """make_sweep's instances for the CPU arm, drawn with the same generator
    calls but without the CUDA library's parameter struct."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_inst):
        n = max(2, int(round(10 ** rng.uniform(2.0, 5.0))) // 2 * 2)
        pair = (3, 1) if rng.random() < 0.5 else (1, 0)
        temp = 10 ** rng.uniform(np.log10(4.0), 4.0)
        b0 = rng.uniform(1.0, 5.0)
        volt = rng.uniform(5.0, 50.0)
        radii = rng.uniform(5e-5, 5e-4, 3)
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        pos = d * rng.random((n, 1)) ** (1.0 / 3.0) * radii
        sp = np.repeat(np.array(pair, np.uint8), n // 2)
        m = np.array([MASS[int(k)] for k in pair]).repeat(n // 2)
        vel = rng.normal(size=(n, 3)) * np.sqrt(KB * temp / m)[:, None]
        out.append((pos, vel, sp, _SweepParams(b0, volt, pair)))
    return out


# ================================================================== long4m
def long_params(learned, n_half=2097152):
    """The long run at scale: 2 x n_half particles (positrons + antiprotons),
    uniform ellipsoid 5e-4 x 5e-4 x 2e-3 m, 100 K, b0 = 5 T, U = 100 V,
    z0 = rho0 = 0.02 m, cooling at 4 K with cooling_scale 10, annihilation at
    1e-6 m with p = 1, FMM energies. learned: the p = 2 FMM plus the learned
    correction with a direct-sum audit every 100 steps and plain p = 6 after
    a failed audit; else plain p = 6."""
    import amk
    kw = dict(seed=42, b0=5.0, trap_voltage=100.0, z0=0.02, rho0=0.02, num_steps=10000,
              populations={"positron": n_half, "antiproton": n_half},
              temperatures={"positron": 100.0, "antiproton": 100.0}, cloud_radii=(5e-4, 5e-4, 2e-3),
              bath_temperature=4.0, cooling_scale=10.0, cooling_enabled=1, coulomb_forces_enabled=1,
              coulomb_method="fast-multipole", fast_multipole_order=6, fast_multipole_theta=0.5,
              energy_method="fast-multipole", annihilation_enabled=1, contact_radius=1e-6,
              annihilation_probability=1.0, fmm_learned=1 if learned else 0, learned_fallback_order=6,
              learned_error_budget=ERROR_BUDGET, learned_audit_interval=100, learned_audit_samples=1024)
    return amk.make_params(**kw)


def long_run(sim, stream, steps, log_every):
    """Steps in chunks of log_every, the FP64 total energy after each chunk
    (outside the timed events); returns (ms, live particle-steps, drift rows)."""
    import torch
    e0 = sim.energy()
    depth = E * 100.0  # the reference's drift scale: the trap depth e |U| (antimatter-kernel.cc:137-142)
    rows = [{"step": 0, "total_J": e0["total"], "fractional_drift": 0.0, "alive": e0["num_active"]}]
    ms, work, done = 0.0, 0.0, 0
    while done < steps:
        k = min(log_every, steps - done)
        a0 = sim.num_alive()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        sim.step(k)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms += ev0.elapsed_time(ev1)
        done += k
        e = sim.energy()
        work += 0.5 * (a0 + e["num_active"]) * k
        rows.append({"step": done, "total_J": e["total"], "fractional_drift": (e["total"] - e0["total"]) / depth,
                     "alive": e["num_active"]})
    return ms, work, rows


def run_long(args):
    import torch
    import amk
    world, rank, local = dist_setup()
    init_nccl(world, local)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    n_half = args.long_n // 2
    out = {}
    for name, learned in (("learned p=2 + MLP, fallback p=6", True), ("plain p=6", False)):
        sim = amk.Simulation(long_params(learned, n_half), device=local)
        sim.init_particles_gpu("uniform")
        stream = torch.cuda.ExternalStream(sim.stream(), device=device)
        entry = {}
        if learned:
            t0 = time.perf_counter()
            loss, samples = sim.fmm_train_correction(0.5, **LEARNED_TRAINING)
            entry["training"] = {"seconds": round(time.perf_counter() - t0, 2), "samples": samples,
                                 "final_loss": loss}
        sampler = ClockSampler(local)
        sampler.start()
        launches0 = sim.kernel_launches()
        ms, work, rows = long_run(sim, stream, args.steps, args.log_every)
        entry.update(value=work / (ms * 1e-3), ms_per_step=ms / args.steps, drift=rows,
                     gpu_launches=sim.kernel_launches() - launches0, clocks=sampler.stop())
        if learned:
            st = sim.fmm_learned_state()
            entry["learned_state"] = st
        out[name] = entry
        sim.close()
    a, b = out["learned p=2 + MLP, fallback p=6"], out["plain p=6"]
    gap = max(abs(x["fractional_drift"] - y["fractional_drift"]) for x, y in zip(a["drift"], b["drift"]))
    if rank == 0:
        line = {"metric": METRIC, "value": a["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": 0, "ms_per_step": a["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (GPU Philox uniform-ellipsoid cloud, seed 42)",
                "config": {"workload": f"long run at scale: N={2 * n_half:,} ({n_half:,} e+ + {n_half:,} pbar), "
                                       "uniform ellipsoid 5e-4 x 5e-4 x 2e-3 m, 100 K, b0=5 T, U=100 V, "
                                       "z0=rho0=0.02 m, cooling (4 K, scale 10), annihilation (1e-6 m, p=1); "
                                       f"{args.steps} of the 10,000 steps, FP64 total-energy drift every "
                                       f"{args.log_every} steps, learned p=2 with p=6 fallback vs plain p=6",
                           "n_particles": 2 * n_half, "log_every": args.log_every,
                           "l2": "not flushed: state of 4 M particles exceeds L2",
                           "parallelism": f"replicas x{world}"},
                "runs": out, "max_drift_gap": gap, "gpu_launches": a["gpu_launches"], "clocks": a["clocks"],
                "roofline": None, "cpu_baseline": None,
                "e2e": None}
        print(json.dumps(line), flush=True)
    finish_dist(world)
    return 0


def run_reference_long(args):
    world, rank, _ = dist_setup()
    if rank == 0:
        print(json.dumps({"impl": "reference", "unavailable": "the 4M long run is measured on the GPU arm only; "
                                                             "the reference's CPU FMM takes minutes per step here"}))
    return 0


# ================================================================== kernels
def phase_ms(sim, fn, phase, reps):
    """Device ms per launch of one library phase (CUDA events the library
    records around it), over `reps` calls of fn after one untimed call."""
    fn()
    sim.synchronize()
    sim.set_profiling(True)
    sim.reset_phase_times()
    for _ in range(reps):
        fn()
    sim.synchronize()
    ms, cnt = sim.phase_times()[phase]
    sim.set_profiling(False)
    return ms / max(cnt, 1), cnt / reps


def run_kernels(args):
    """The HBM-bound per-particle kernels and the MLP's tensor-core forward,
    each timed live in its library phase and set against its roofline:
    the Boris push with cooling (4,194,304 particles), the radix sort and
    octree build of an FMM evaluation (4,194,304 positrons), the
    annihilation contact search and matching (4,194,304 particles, 1e-6 m)
    and the learned correction's MLP forward (1,048,576 samples). This is
    also the command the kernels' ncu captures run."""
    import torch
    import amk
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    hbm, hbm_src = measured_peak("hbm_gbs", 6650.0)
    bf16, bf16_src = measured_peak("bf16_tflops", 1590.0)
    n = args.long_n
    out = {}
    p = long_params(False, n // 2)
    with amk.Simulation(p, device=local) as sim:
        sim.init_particles_gpu("uniform")
        ms, per = phase_ms(sim, sim.push, "push", args.steps)
        bytes_ = 165.0 * n  # x, v read and written, F read and zeroed, q, m, id, alive
        out["push_kernel"] = {"ms": ms, "algorithmic_bytes": bytes_, "achieved_gbs": bytes_ / (ms * 1e-3) / 1e9,
                              "frac": bytes_ / (ms * 1e-3) / 1e9 / hbm, "launches_per_call": per,
                              "unit": "165 B per particle-step: x, v read + written (96), F read + zeroed (48), "
                                      "q, m (16), id (4), alive (1)"}
        ms, per = phase_ms(sim, lambda: sim.annihilate(), "annihilation", args.steps)
        bytes_ = (24.0 + 2 + 12 + 32 * 8 + 24 * 27 / 8) * n
        out["annihilation (cell list, contact_kernel, matching)"] = {
            "ms": ms, "algorithmic_bytes": bytes_, "achieved_gbs": bytes_ / (ms * 1e-3) / 1e9,
            "frac": bytes_ / (ms * 1e-3) / 1e9 / hbm,
            "unit": "per particle: positions (24), species + alive (2), cell key + index written (12), 8 radix "
                    "passes x 32 B, neighbour positions of the 27 cells read once per 8 particles (81)"}
    pos, vel, sp = tree_cloud(n)
    with amk.Simulation(tree_params(n, dict(coulomb_method="fast-multipole", fast_multipole_order=4,
                                            fast_multipole_theta=0.5)), device=local) as sim:
        sim.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], sp)
        sim.coulomb()
        sim.synchronize()
        sim.set_profiling(True)
        sim.reset_phase_times()
        for _ in range(args.steps):
            sim.coulomb()
        sim.synchronize()
        ph = sim.phase_times()
        sim.set_profiling(False)
        nodes = sim.fmm_stats()["cells"]
        sort_ms = ph["sort"][0] / max(ph["sort"][1], 1)
        tree_ms = ph["tree"][0] / max(ph["tree"][1], 1) - sort_ms  # the tree phase encloses the sort
        sb = 256.0 * n
        tb = 100.0 * n + 78.0 * nodes
        out["radix sort (hist_kernel, scan, scatter_staged_kernel)"] = {
            "ms": sort_ms, "algorithmic_bytes": sb, "achieved_gbs": sb / (sort_ms * 1e-3) / 1e9,
            "frac": sb / (sort_ms * 1e-3) / 1e9 / hbm,
            "unit": "256 B per key: 8 passes of 8 B key read (histogram) + 12 B read + 12 B written (scatter)"}
        out["octree build (tree_*_kernel)"] = {
            "ms": tree_ms, "algorithmic_bytes": tb, "achieved_gbs": tb / (tree_ms * 1e-3) / 1e9,
            "frac": tb / (tree_ms * 1e-3) / 1e9 / hbm, "nodes": nodes,
            "unit": "100 B per source (keys, key-prefix lengths, leaf depths, counts, gathered position + charge, "
                    "source written) + 78 B per node (centre, children, range, meta, parent)"}
    m = 1 << 20
    with amk.Simulation(tree_params(m, dict(coulomb_method="fast-multipole", fast_multipole_order=2,
                                            fast_multipole_theta=0.5, fmm_learned=1,
                                            learned_audit_interval=0)), device=local) as sim:
        sim.set_particles(pos[:m, 0], pos[:m, 1], pos[:m, 2], vel[:m, 0], vel[:m, 1], vel[:m, 2], sp[:m])
        sim.fmm_train_correction(0.5, sample_leaves=256, steps=20, batch=1024, lr=1e-3)
        ms, per = phase_ms(sim, sim.coulomb, "mlp", args.steps)
        flops = 2.0 * (35 * 128 + 2 * 128 * 128 + 128 * 3) * m
        out["mlp_forward_tc_kernel"] = {
            "ms": ms, "algorithmic_flops": flops, "achieved_tflops": flops / (ms * 1e-3) / 1e12,
            "frac": flops / (ms * 1e-3) / 1e12 / bf16,
            "unit": "2 (35x128 + 2x128x128 + 128x3) flop per sample (unpadded), 1,048,576 samples"}
    if rank == 0:
        print(json.dumps({"workload": "kernels", "steps": args.steps, "peaks": {"hbm_gbs": [hbm, hbm_src],
                                                                                "bf16_tflops": [bf16, bf16_src]},
                          "kernels": out}), flush=True)
    return 0


# ================================================================== main
WORKLOADS = {"tree1m": (run_tree, run_reference_tree), "direct65k": (run_direct, run_reference_direct),
             "sweep512": (run_sweep, run_reference_sweep), "long4m": (run_long, run_reference_long),
             "kernels": (run_kernels, run_reference_long)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["amk", "reference"], default="amk")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="tree1m")
    ap.add_argument("--cpu-baseline", type=int, default=1, help="time the reference's CPU leg (rank 0, N=1)")
    ap.add_argument("--cpu-sample", type=int, default=8192, help="targets of the direct workload's CPU leg")
    ap.add_argument("--ref-sample", type=int, default=65536,
                    help="particles of the tree workload's reference sample (the cloud's first ones)")
    ap.add_argument("--ref-sample-direct", type=int, default=512,
                    help="targets per step of the direct workload's reference arm")
    ap.add_argument("--ref-pairs", type=float, default=2e9,
                    help="particle pairs per step of the sweep workload's reference sample")
    ap.add_argument("--audit-samples", type=int, default=4096, help="particles audited against FP64")
    ap.add_argument("--method-steps", type=int, default=5, help="timed steps of each method in the table")
    ap.add_argument("--autotune", type=int, default=1,
                    help="tree workload: also time the FMM configuration the library's autotuner picks")
    ap.add_argument("--sweep-ratio", type=int, default=1,
                    help="tree workload: also measure the sweep's batched / one-at-a-time ratio")
    ap.add_argument("--sweep-steps", type=int, default=20, help="batched steps of the sweep ratio")
    ap.add_argument("--serial-steps", type=int, default=3, help="steps of the one-at-a-time comparison")
    ap.add_argument("--instances", type=int, default=512, help="trap instances of the sweep")
    ap.add_argument("--tree-n", type=int, default=1 << 20, help="particles of the tree workload")
    ap.add_argument("--tree-methods", default="", help="comma-separated subset of the tree workload's methods")
    ap.add_argument("--fmm-leaf", type=int, default=0,
                    help="leaf capacity of the table's FMM methods (0: the library's default, 32)")
    ap.add_argument("--long-n", type=int, default=1 << 22, help="particles of the long run")
    ap.add_argument("--log-every", type=int, default=100, help="steps between energy logs of the long run")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)  # at least three untimed warm-up steps
    amk_fn, ref_fn = WORKLOADS[args.workload]
    return (ref_fn if args.impl == "reference" else amk_fn)(args)


if __name__ == "__main__":
    sys.exit(main())
