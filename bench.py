#!/usr/bin/env python
"""Benchmark of the B200 particle path; prints ONE JSON line on rank 0.

Workload (default ``direct65k``): the plain direct all-pairs Coulomb run --
N = 65,536 (32,768 positrons + 32,768 antiprotons, real charges and masses),
uniform ellipsoidal cloud with radii 2e-4 x 2e-4 x 5e-4 m drawn by the
reference's own generator (seed 42), Maxwellian velocities at 10 K, b0 = 3 T,
trap_voltage = 50 V, z0 = rho0 = 0.01 m, dt from the reference's rule
(2.977e-12 s), FP32 pair arithmetic with compensated accumulation and FP64
state, cooling and annihilation off. One bench step = one simulation step
(all-pairs force -> Boris push) of the whole cloud.

``value`` is particle-steps/s over all ranks with the state resident in HBM
(device-timed with CUDA events on the library's stream, L2 flushed by a
256 MiB write between steps, the flush outside the per-step events). ``e2e``
is the same metric through the C ABI with host buffers: every step uploads
x, v from pinned host memory (amk_update_state), steps, and reads x, v and
the alive flags back (amk_get_particles).

``--impl reference`` times the reference's own CPU code for the same step on
the host cores (its Barnes-Hut tree at theta = 0, i.e. the exact all-pairs
sum, compiled from the reference sources into oracle/_ref, plus the FP64
push restatement), on a bounded sample of targets per step.

Multi-GPU: the single-instance run does not shard (replicas only); under
torchrun every rank runs its own replica and ``value`` sums them over the
slowest rank's time.
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


def workload_direct65k():
    import amk
    p = amk.make_params(
        seed=42, b0=3.0, trap_voltage=50.0, z0=0.01, rho0=0.01, num_steps=1000,
        populations={"antiproton": 32768, "positron": 32768},
        temperatures={"antiproton": 10.0, "positron": 10.0},
        cloud_radii=(2e-4, 2e-4, 5e-4), bath_temperature=0.0, cooling_scale=0.0,
        cooling_enabled=0, coulomb_forces_enabled=1, coulomb_method="allpairs",
        energy_method="allpairs", annihilation_enabled=0)
    config = {"workload": "direct all-pairs Coulomb + Boris push, N=65,536 "
                          "(32,768 e+ + 32,768 pbar), uniform ellipsoid 2e-4 x 2e-4 x 5e-4 m, "
                          "10 K Maxwellian, b0=3 T, U=50 V, z0=rho0=0.01 m, dt=2.977e-12 s",
              "n_particles": 65536, "solver": "allpairs (tiled FP32, double-float positions, "
                                                  "compensated accumulation)",
              "state_precision": "fp64 positions/velocities", "cooling": False,
              "annihilation": False, "seed": 42,
              "l2": "flushed between steps by a 256 MiB write (inputs 6.5 MB < L2)"}
    return p, config


KB = 1.380649e-23
MASS = {0: 1.67262192369e-27, 1: 9.1093837015e-31, 3: 9.1093837015e-31, 4: 1.67262192369e-27}


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


WORKLOADS = {"direct65k": workload_direct65k, "sweep512": None, "tree1m": None}


def tree_cloud(n=1 << 20, seed=42):
    """N positrons, Gaussian cloud sigma 1e-4, 1e-4, 3e-4 m, 5 K Maxwellian."""
    rng = np.random.default_rng(seed)
    pos = rng.normal(0.0, 1.0, (n, 3)) * np.array([1e-4, 1e-4, 3e-4])
    vel = rng.normal(0.0, 1.0, (n, 3)) * np.sqrt(KB * 5.0 / MASS[1])
    return pos, vel, np.ones(n, np.uint8)


TREE_METHODS = [
    ("allpairs", dict(coulomb_method="allpairs")),
    ("barnes-hut theta=0.7", dict(coulomb_method="barnes-hut", barnes_hut_theta=0.7)),
    ("fmm p=4 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=4, fast_multipole_theta=0.5)),
    ("fmm p=6 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=6, fast_multipole_theta=0.5)),
    ("fmm p=7 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=7, fast_multipole_theta=0.5)),
    ("fmm p=8 theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=8, fast_multipole_theta=0.5)),
    ("learned p=2 + MLP theta=0.5", dict(coulomb_method="fast-multipole", fast_multipole_order=2,
                                        fast_multipole_theta=0.5, fmm_learned=1, learned_audit_interval=0)),
]


# DRAM traffic (read + write) per launch of the FMM's M2L class-product kernel,
# by order: from ncu captures of one launch (one chunk of at most 4 GiB of
# per-pair products; launches at N = 1,048,576 process chunks of the same size).
FMM_PRODUCT_TRAFFIC = {
    7: (5.18e9, "ncu dram__bytes_read.sum + dram__bytes_write.sum of m2l_class_mma_kernel<7>, mean of two launches "
                "of 4.47 M pairs each (0.89 / 1.10 GB read + 4.18 GB written: the per-pair products), "
                "profiles/m2l_class_mma_kernel_tree1m.md"),
    8: (5.17e9, "ncu dram__bytes_read.sum + dram__bytes_write.sum of m2l_class_mma_kernel<8>, mean of two launches "
                "of 3.25 M pairs each (0.92 GB read + 4.26 GB written: the per-pair products), "
                "profiles/m2l_class_mma_kernel_tree1m.md"),
}


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


# ------------------------------------------------------------------ CPU legs
def cpu_reference_step_time(x, y, z, q, m, n_sample, seed=0):
    """Reference CPU step on a bounded sample: the reference's Barnes-Hut tree
    at theta = 0 (exact all-pairs) over all N sources, walked for n_sample
    targets and extrapolated to N, plus the FP64 push of all N particles.
    Returns (seconds per full step, kind, sampled target ids, sampled forces)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_lib as O
    n = len(x)
    rng = np.random.default_rng(seed)
    targets = np.sort(rng.choice(n, n_sample, replace=False))
    if O.ref_available():
        kind = "reference"
        t0 = time.perf_counter()
        O.ref_bh_forces_subset(x, y, z, q, 0.0, targets[:1], 8)
        t_build = time.perf_counter() - t0
        t0 = time.perf_counter()
        f = O.ref_bh_forces_subset(x, y, z, q, 0.0, targets, 8)
        t_walk = max(time.perf_counter() - t0 - t_build, 1e-9)
    else:
        kind = "port"
        t_build = 0.0
        t0 = time.perf_counter()
        f = O.allpairs_subset(x, y, z, q, targets)
        t_walk = time.perf_counter() - t0
    state = dict(x=x.copy(), y=y.copy(), z=z.copy(), vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n),
                 q=q, m=m, alive=np.ones(n, np.uint8))
    t0 = time.perf_counter()
    O.boris_push(state, np.zeros(n), np.zeros(n), np.zeros(n), 3.0, 50.0, 0.01, 0.01, 2.977e-12, True)
    t_push = time.perf_counter() - t0
    return t_build + t_walk * n / n_sample + t_push, kind, targets, f


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    import amk
    p, config = WORKLOADS[args.workload]()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_lib as O
    pops = {"antiproton": 32768, "positron": 32768}
    pos = O.initial_positions(pops, [2e-4, 2e-4, 5e-4], 42)
    sp = O.species_column(pops)
    m, q = O.species_props(sp)
    x, y, z = pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()
    sample = args.ref_sample
    times = []
    kind = "reference"
    for k in range(args.warmup + args.steps):
        t, kind, _, _ = cpu_reference_step_time(x, y, z, q, m, sample, seed=k)
        if k >= args.warmup:
            times.append(t)
    t_step = float(np.mean(times))
    value = len(x) / t_step
    cores = os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference initial-condition generator, seed 42)", "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"per step: tree over all {len(x)} sources, theta=0 walks for "
                                       f"{sample} sampled targets extrapolated to {len(x)}, FP64 "
                                       f"push of all {len(x)}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ batched sweep
def cpu_sweep_step_time(insts, n_sample=64):
    """Reference CPU step of every instance on a bounded sample: the
    reference's Barnes-Hut tree at theta = 0 (exact all-pairs) built over
    each instance's sources and walked for up to n_sample targets,
    extrapolated to the instance, plus the FP64 push of every particle."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_lib as O
    total = 0.0
    kind = "reference" if O.ref_available() else "port"
    for pos, vel, sp, p in insts:
        n = len(pos)
        m, q = O.species_props(sp)
        x, y, z = pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()
        k = min(n, n_sample)
        targets = np.arange(k) * (n // k)
        t_build = 0.0
        if kind == "reference":
            t0 = time.perf_counter()
            O.ref_bh_forces_subset(x, y, z, q, 0.0, targets[:1], 8)  # tree build + one walk
            t_build = time.perf_counter() - t0
            t0 = time.perf_counter()
            O.ref_bh_forces_subset(x, y, z, q, 0.0, targets, 8)
            t_walk = max(time.perf_counter() - t0 - t_build, 1e-9)
        else:
            t0 = time.perf_counter()
            O.allpairs_subset(x, y, z, q, targets)
            t_walk = time.perf_counter() - t0
        state = dict(x=x, y=y, z=z, vx=vel[:, 0].copy(), vy=vel[:, 1].copy(), vz=vel[:, 2].copy(),
                     q=q, m=m, alive=np.ones(n, np.uint8))
        t0 = time.perf_counter()
        O.boris_push(state, np.zeros(n), np.zeros(n), np.zeros(n), p.b0, p.trap_voltage, p.z0, p.rho0,
                     p.dt, True)
        t_push = time.perf_counter() - t0
        total += t_build + t_walk * n / k + t_push
    return total, kind


def run_sweep(args):
    """Batched 512-instance sweep: batched step (one persistent all-pairs
    launch, CUDA-graph chunks) against the same instances stepped one at a
    time with the single-instance kernels."""
    import torch
    import amk
    world, rank, local = dist_setup()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    # every rank runs its own sweep of 512 instances (seeded by rank): the
    # instances are independent, so the sweep shards with no collective
    insts = make_sweep(n_inst=args.instances, seed=2024 + rank, method_split=None)
    n_total = int(sum(len(i[0]) for i in insts))
    sim = amk.Simulation(device=local)
    load_sweep(sim, insts)
    # per-instance method by measurement under the 1e-5 RMS force-error budget
    t0 = time.perf_counter()
    methods = sim.batch_autotune(error_budget=1e-5, samples=256)
    tune_s = time.perf_counter() - t0
    names = {-1: "none", 0: "cutoff", 1: "barnes-hut", 2: "fmm", 3: "allpairs"}
    method_counts = {names[int(m)]: int((methods == m).sum()) for m in np.unique(methods)}
    chunk = min(100, args.steps)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def live():
        return int(sim.batch_status()["alive"].sum())

    def live_rate(ms, steps, before, after):
        # particle-steps/s over the live particles (annihilated ones do no work)
        return world * 0.5 * (before + after) * steps / (ms * 1e-3)

    def timed(fn):
        # events on the stream of the context in use (contexts are replaced below)
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

    # warm-up: plain steps (the first is the staggered one), then one chunk to
    # capture and instantiate the graph outside the timed region
    sim.batch_step(args.warmup)
    sim.batch_step(chunk, graph_chunk=chunk)
    sim.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = sim.kernel_launches()
    live0 = live()
    ms = timed(lambda: sim.batch_step(args.steps, graph_chunk=chunk))
    live1 = live()
    launches = sim.kernel_launches() - launches0
    clocks = sampler.stop()
    ms = max_over_ranks(ms, world, device)
    value = live_rate(ms, args.steps, live0, live1)

    # per-phase device time (profiling runs plain steps, no graph)
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
    roofline = {"bound": "fp32", "kernel": "batch_allpairs_kernel", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": 116.2e6 * n_total / 1380664,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of batch_allpairs_kernel "
                                  "on the 64-instance case (116.2 MB for 1,380,664 particles, "
                                  "profiles/batch_allpairs_kernel_sweep.md), scaled by particle count (the "
                                  "staged particle data read once plus the force writes)",
                "peak_source": "measured in this run: FFMA probe kernel over all SMs (2 flop/FFMA)",
                "flops_per_launch": 20.0 * pairs,
                "flop_convention": "20 flop per pair interaction x sum_i A_i(A_i-1), A_i the live "
                                   "particles of all-pairs instance i",
                "avg_launch_ms": ap_avg,
                "phase_ms_per_step": {k: v[0] / prof_steps for k, v in phases.items() if v[1]}}

    # baseline: the same instances one at a time with the single-instance kernels
    serial_steps = max(1, min(args.steps, args.serial_steps))
    sim.batch_step(1, serial=True)  # untimed: grows the single-instance scratch to its largest size
    s_live0 = live()
    serial_ms = max_over_ranks(timed(lambda: sim.batch_step(serial_steps, serial=True)), world, device)
    serial_value = live_rate(serial_ms, serial_steps, s_live0, live())
    sim.close()
    # the sweep's own method split (FMM p=4 from 8,192 particles), both ways
    split = make_sweep(n_inst=args.instances, seed=2024 + rank, method_split=8192, order=4)
    sim = amk.Simulation(device=local)
    load_sweep(sim, split)
    sim.batch_step(args.warmup)
    p_live0 = live()
    split_ms = max_over_ranks(timed(lambda: sim.batch_step(serial_steps)), world, device)
    split_value = live_rate(split_ms, serial_steps, p_live0, live())
    sim.batch_step(1, serial=True)
    p_live0 = live()
    split_serial_ms = max_over_ranks(timed(lambda: sim.batch_step(serial_steps, serial=True)), world, device)
    split_serial_value = live_rate(split_serial_ms, serial_steps, p_live0, live())

    # end to end through the C ABI with host buffers (one step per call)
    L = amk.lib()
    sim.close()
    sim = amk.Simulation(device=local)
    load_sweep(sim, insts)
    sim.batch_step(args.warmup)
    host = {k: torch.empty(n_total, dtype=torch.float64, pin_memory=True) for k in
            ("x", "y", "z", "vx", "vy", "vz")}
    alive = torch.empty(n_total, dtype=torch.uint8, pin_memory=True)
    order = ("x", "y", "z", "vx", "vy", "vz")
    ptr = {k: v.data_ptr() for k, v in host.items()}
    amk.check(L.amk_get_particles(sim.handle, *[_dp(ptr[k]) for k in order],
                                  C.cast(C.c_void_p(alive.data_ptr()), C.POINTER(C.c_uint8))))
    e2e_steps = max(1, min(args.steps, 10))

    def e2e_loop():
        for _ in range(e2e_steps):
            sim.update_state(*[ptr[k2] for k2 in order])
            sim.batch_step(1)
            amk.check(L.amk_get_particles(sim.handle, *[_dp(ptr[k2]) for k2 in order],
                                          C.cast(C.c_void_p(alive.data_ptr()), C.POINTER(C.c_uint8))))
    e_live0 = live()
    e2e_ms = max_over_ranks(timed(e2e_loop), world, device)
    e2e = {"value": live_rate(e2e_ms, e2e_steps, e_live0, live()), "unit": UNIT,
           "h2d_bytes_per_step": 6 * 8 * n_total, "d2h_bytes_per_step": 6 * 8 * n_total + n_total,
           "steps": e2e_steps,
           "api": "amk_update_state + amk_batch_step + amk_get_particles (pinned host buffers)"}
    status = sim.batch_status()
    sim.close()

    cpu = None
    if rank == 0 and world == 1:
        t_cpu, kind = cpu_sweep_step_time(insts)
        cpu = {"value": n_total / t_cpu, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
               "sample": "per instance: reference Barnes-Hut theta=0 tree over all its sources walked "
                         "for 64 evenly spaced targets (extrapolated), + FP64 push of all particles; "
                         "all instances, OpenMP on all host cores"}
    if rank == 0:
        sizes = np.array([len(i[0]) for i in insts])
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic (seeded sweep generator)",
                "config": {"workload": f"batched sweep: {len(insts)} trap instances, N_i log-uniform 1e2..1e5 "
                                       f"(total {n_total:,}), e-/e+ or e+/pbar 1:1, T 4..1e4 K, b0 1..5 T, "
                                       "U 5..50 V, radii 5e-5..5e-4 m, cooling (4 K) and annihilation "
                                       "(5e-6 m, p=0.5) on",
                           "solver": "per-instance method chosen by amk_batch_autotune under a 1e-5 "
                                     "RMS force-error budget; all-pairs instances share one persistent "
                                     "launch (cost-ordered work queue); FP64 state",
                           "autotune": {"methods": method_counts, "seconds": round(tune_s, 2)},
                           "graph_chunk": chunk, "instances": len(insts), "n_particles": n_total,
                           "live_particles_timed": [live0, live1],
                           "rate_counts": "live (not yet annihilated) particles, mean of the timed "
                                          "window's start and end",
                           "instance_sizes": {"min": int(sizes.min()), "median": int(np.median(sizes)),
                                              "max": int(sizes.max())},
                           "l2": "not flushed: state of 7.4 M particles (> 700 MB) exceeds L2",
                           "parallelism": f"dp{world}: one {len(insts)}-instance sweep per GPU, no collective"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks,
                "one_at_a_time": {"value": serial_value, "steps": serial_steps,
                                  "ms_per_step": serial_ms / serial_steps,
                                  "speedup_batched": value / serial_value,
                                  "api": "amk_batch_step(serial=1): each instance through the "
                                         "single-instance kernels, one after another"},
                "method_split_8192_fmm_p4": {
                    "batched_value": split_value,
                    "one_at_a_time_value": split_serial_value,
                    "note": "all-pairs below 8,192 particles, FMM p=4 theta=0.5 above (RMS error "
                            "about 7e-5, above the 1e-5 bar); per-instance FMM calls synchronise "
                            "with the host, so no graphs"},
                "contact_overflow": bool(status["overflow"])}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_reference_tree(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    pos, _, _ = tree_cloud(args.tree_n)
    n = len(pos)
    x, y, z = pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()
    q = np.full(n, E)
    m = np.full(n, MASS[1])
    times = []
    kind = "reference"
    for k in range(args.warmup + args.steps):
        t, kind, _, _ = cpu_reference_step_time(x, y, z, q, m, args.ref_sample, seed=k)
        if k >= args.warmup:
            times.append(t)
    t_step = float(np.mean(times))
    value = n / t_step
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian cloud)",
            "config": {"workload": f"tree solvers at N={n:,} positrons (exact force)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
                             "sample": f"per step: theta=0 tree over all {n} sources, {args.ref_sample} targets "
                                       f"walked (extrapolated), FP64 push of all"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_sweep(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    insts = make_sweep(n_inst=args.instances, seed=2024, method_split=None)
    n_total = int(sum(len(i[0]) for i in insts))
    times = []
    kind = "reference"
    for k in range(args.warmup + args.steps):
        t, kind = cpu_sweep_step_time(insts, n_sample=16)
        if k >= args.warmup:
            times.append(t)
    t_step = float(np.mean(times))
    value = n_total / t_step
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded sweep generator)",
            "config": {"workload": f"batched sweep: {len(insts)} trap instances, {n_total:,} particles"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
                             "sample": "per instance and step: theta=0 tree over all sources, 16 "
                                       "targets walked (extrapolated), FP64 push of all"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ tree solvers at 1M
def run_tree(args):
    """N = 1,048,576 positrons: every Coulomb method timed per step (force +
    push) and audited against the FP64 exact sum; `value` is the fastest
    method whose RMS relative force error is within 1e-5."""
    import torch
    import amk
    world, rank, local = dist_setup()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    pos, vel, sp = tree_cloud(args.tree_n)
    n = len(pos)
    steps = max(1, min(args.steps, 5))
    results = {}
    best = None
    methods = [m for m in TREE_METHODS if not args.tree_methods or m[0] in args.tree_methods.split(",")]
    if not methods:
        raise SystemExit(f"--tree-methods: none of {[m[0] for m in TREE_METHODS]}")
    for name, over in methods:
        kw = dict(seed=42, b0=1.0, trap_voltage=10.0, z0=0.01, rho0=0.01, num_steps=500,
                  populations={"positron": n}, temperatures={"positron": 5.0}, cloud_radii=(1e-4, 1e-4, 3e-4),
                  bath_temperature=0.0, cooling_scale=0.0, cooling_enabled=0, coulomb_forces_enabled=1,
                  energy_method="allpairs", annihilation_enabled=0)
        kw.update(over)
        sim = amk.Simulation(amk.make_params(**kw), device=local)
        sim.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], sp)
        entry = {}
        if over.get("fmm_learned"):
            t0 = time.perf_counter()
            loss, samples = sim.fmm_train_correction(0.5, sample_leaves=4096, steps=2000, batch=4096, lr=1e-3)
            entry["training"] = {"seconds": round(time.perf_counter() - t0, 2), "samples": samples,
                                 "final_loss": loss}
        sim.coulomb()
        rms, mx = sim.force_error(1024)
        entry.update({"rms_rel": rms, "max_rel": mx, "meets_1e-5": bool(rms <= 1e-5)})
        stream = torch.cuda.ExternalStream(sim.stream(), device=device)
        sim.step(max(1, args.warmup))
        sim.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        sim.step(steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        entry.update(ms_per_step=ms, value=n / (ms * 1e-3), steps=steps)
        sim.set_profiling(True)
        sim.reset_phase_times()
        sim.step(1)
        sim.synchronize()
        entry["phase_ms"] = {k: round(v[0], 3) for k, v in sim.phase_times().items() if v[1]}
        sim.set_profiling(False)
        results[name] = entry
        if entry["meets_1e-5"] and (best is None or entry["value"] > results[best]["value"]):
            best = name
        sim.close()
    # the winner again: roofline of its dominant kernel, e2e through the C ABI
    name = best if best is not None else methods[0][0]
    over = dict(TREE_METHODS)[name]
    kw = dict(seed=42, b0=1.0, trap_voltage=10.0, populations={"positron": n}, cooling_enabled=0,
              energy_method="allpairs", annihilation_enabled=0)
    kw.update(over)
    sim = amk.Simulation(amk.make_params(**kw), device=local)
    sim.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], sp)
    sim.step(1)
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = sim.kernel_launches()
    stream = torch.cuda.ExternalStream(sim.stream(), device=device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    sim.step(steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = sim.kernel_launches() - launches0
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / steps
    value = n / (ms * 1e-3)
    roofline = None
    if over["coulomb_method"] == "allpairs":
        sim.set_profiling(True)
        sim.reset_phase_times()
        sim.step(1)
        sim.synchronize()
        ap_ms, ap_n = sim.phase_times()["allpairs"]
        sim.set_profiling(False)
        peak = sim.measure_fp32_peak()
        achieved = 20.0 * n * (n - 1) / (ap_ms / ap_n * 1e-3) / 1e12
        roofline = {"bound": "fp32", "kernel": "allpairs_kernel", "achieved": achieved, "peak": peak,
                    "unit": "TFLOP/s", "frac": achieved / peak, "traffic": 3.276e6 * n / 65536,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of allpairs_kernel at "
                                      "N = 65,536 (3.276 MB, profiles/allpairs_kernel_direct65k.md), scaled by N "
                                      "(sources are read from DRAM once per launch and re-read from L2)",
                    "peak_source": "measured in this run: FFMA probe kernel over all SMs (2 flop/FFMA)",
                    "flop_convention": "20 flop per pair interaction x N(N-1) pairs",
                    "avg_launch_ms": ap_ms / ap_n}
    elif over["coulomb_method"] == "fast-multipole" and not over.get("fmm_learned"):
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
        peak = sim.measure_fp64_peak()
        achieved = 2.0 * nm * nm * st["m2l_class_pairs"] / (prod_ms * 1e-3) / 1e12
        traffic = FMM_PRODUCT_TRAFFIC.get(p_)
        roofline = {"bound": "fp64 tensor", "kernel": f"m2l_class_mma_kernel<{p_}>", "achieved": achieved,
                    "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                    "traffic": None if traffic is None else traffic[0],
                    "traffic_source": None if traffic is None else traffic[1],
                    "peak_source": "measured in this run: mma.m8n8k4 FP64 probe kernel over all SMs "
                                   "(512 flop per warp instruction)",
                    "flop_convention": f"2 n_m^2 flop (n_m = {nm}) per M2L pair evaluated as a class product "
                                       f"({st['m2l_class_pairs']:,} of {st['m2l_pairs']:,} pairs; the rest take "
                                       "the per-pair path)",
                    "avg_launch_ms": prod_ms / max(1, prod_n), "launches_per_step": prod_n,
                    "m2l_phase_ms": ph["fmm_m2l"][0], "classes": st["m2l_classes"]}
    host = {k: torch.empty(n, dtype=torch.float64, pin_memory=True) for k in ("x", "y", "z", "vx", "vy", "vz")}
    alive = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    order = ("x", "y", "z", "vx", "vy", "vz")
    ptr = {k: v.data_ptr() for k, v in host.items()}
    L = amk.lib()
    amk.check(L.amk_get_particles(sim.handle, *[_dp(ptr[k]) for k in order],
                                  C.cast(C.c_void_p(alive.data_ptr()), C.POINTER(C.c_uint8))))
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        sim.update_state(*[ptr[k] for k in order])
        sim.step(1)
        amk.check(L.amk_get_particles(sim.handle, *[_dp(ptr[k]) for k in order],
                                      C.cast(C.c_void_p(alive.data_ptr()), C.POINTER(C.c_uint8))))
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = ev0.elapsed_time(ev1)
    e2e = {"value": n * steps / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 48 * n,
           "d2h_bytes_per_step": 49 * n, "steps": steps,
           "api": "amk_update_state + amk_step + amk_get_particles (pinned host buffers)"}
    st = sim.get_particles()
    sim.close()
    cpu = None
    if rank == 0 and world == 1:
        q = np.full(n, E)
        m = np.full(n, MASS[1])
        t_step, kind, _, _ = cpu_reference_step_time(st["x"], st["y"], st["z"], q, m, args.cpu_sample)
        cpu = {"value": n / t_step, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
               "sample": f"reference Barnes-Hut theta=0 (exact all-pairs) tree over all {n} sources walked for "
                         f"{args.cpu_sample} sampled targets, extrapolated to {n}, + FP64 push of all {n}"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32" if over["coulomb_method"] == "allpairs" else "f64",
            "data": "synthetic (seeded Gaussian cloud)",
            "config": {"workload": f"tree solvers at N={n:,} positrons, Gaussian sigma 1e-4 x 1e-4 x 3e-4 m, "
                                   "5 K Maxwellian, b0=1 T, U=10 V; value = fastest method within 1e-5 RMS "
                                   "relative force error vs the FP64 exact sum (1,024 audited particles)",
                       "chosen": name, "methods": results,
                       "l2": "not flushed: state of 1 M particles (> 100 MB) exceeds L2",
                       "parallelism": "replicas x1 (single instance)"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def run_amk(args):
    import torch
    import amk
    world, rank, local = dist_setup()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    p, config = WORKLOADS[args.workload]()
    sim = amk.Simulation(p, device=local)
    sim.init_particles()
    n = sim.num_particles()
    stream = torch.cuda.ExternalStream(sim.stream(), device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    def flush_l2(k):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # ---------------- warm-up
    for k in range(args.warmup):
        sim.step(1)
        flush_l2(k)
    sim.synchronize()

    # ---------------- timed region (resident state)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = sim.kernel_launches()
    for k in range(args.steps):
        starts[k].record(stream)
        sim.step(1)
        ends[k].record(stream)
        flush_l2(k)
    torch.cuda.synchronize()
    barrier()
    launches = sim.kernel_launches() - launches0
    clocks = sampler.stop()
    total_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    total_ms = max_over_ranks(total_ms, world, device)
    value = world * n * args.steps / (total_ms * 1e-3)

    # ---------------- roofline of the dominant kernel (live phase events)
    prof_steps = min(args.steps, 50)
    sim.set_profiling(True)
    sim.reset_phase_times()
    for k in range(prof_steps):
        sim.step(1)
        flush_l2(k)
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

    # ---------------- end to end through the C ABI with host buffers
    L = amk.lib()
    host = {k: torch.empty(n, dtype=torch.float64, pin_memory=True) for k in
            ("x", "y", "z", "vx", "vy", "vz")}
    alive = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    ptr = {k: v.data_ptr() for k, v in host.items()}
    order = ("x", "y", "z", "vx", "vy", "vz")
    amk.check(L.amk_get_particles(sim.handle, *[_dp(ptr[k]) for k in order],
                                  C.cast(C.c_void_p(alive.data_ptr()), C.POINTER(C.c_uint8))))
    e2e_steps = args.steps
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(e2e_steps):
        sim.update_state(*[ptr[k2] for k2 in order])
        sim.step(1)
        amk.check(L.amk_get_particles(sim.handle, *[_dp(ptr[k2]) for k2 in order],
                                      C.cast(C.c_void_p(alive.data_ptr()), C.POINTER(C.c_uint8))))
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1), world, device)
    e2e_value = world * n * e2e_steps / (e2e_ms * 1e-3)
    e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 6 * 8 * n,
           "d2h_bytes_per_step": 6 * 8 * n + n, "steps": e2e_steps,
           "api": "amk_update_state + amk_step + amk_get_particles (pinned host buffers)"}

    # ---------------- CPU baseline + force check (rank 0, one GPU only)
    cpu = None
    err = None
    if rank == 0 and world == 1:
        st = sim.get_particles()
        sim.coulomb_allpairs()
        fx, fy, fz = sim.get_forces()
        q = np.where(np.asarray(_species(sim, p)) == 1, E, -E)
        m = np.where(np.asarray(_species(sim, p)) == 1, 9.1093837015e-31, 1.67262192369e-27)
        t_step, kind, targets, fref = cpu_reference_step_time(st["x"], st["y"], st["z"], q, m,
                                                              args.cpu_sample)
        cpu = {"value": n / t_step, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
               "sample": f"reference Barnes-Hut theta=0 (exact all-pairs) tree over all {n} "
                         f"sources walked for {args.cpu_sample} sampled targets, extrapolated to "
                         f"{n}, + FP64 push of all {n}; OpenMP on all host cores"}
        num = np.sqrt((fx[targets] - fref[0]) ** 2 + (fy[targets] - fref[1]) ** 2 +
                      (fz[targets] - fref[2]) ** 2)
        den = np.sqrt(fref[0] ** 2 + fref[1] ** 2 + fref[2] ** 2)
        rel = num / den
        err = {"rms_rel": float(np.sqrt(np.mean(rel ** 2))), "max_rel": float(np.max(rel)),
               "targets": int(len(targets)), "against": f"{kind} FP64 exact sum"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic (reference initial-condition generator, seed 42)",
                "config": dict(config, parallelism=f"replicas x{world} (single instance does not shard)"),
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks, "force_error_vs_fp64": err}
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def _species(sim, p):
    # species in creation order: populations in enum order (antiproton, positron)
    out = []
    for i in sorted(range(p.n_species), key=lambda k: p.species[k]):
        out += [p.species[i]] * p.populations[i]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["amk", "reference"], default="amk")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="direct65k")
    ap.add_argument("--cpu-sample", type=int, default=8192,
                    help="targets walked by the CPU baseline leg")
    ap.add_argument("--ref-sample", type=int, default=256,
                    help="targets walked per step by the reference arm")
    ap.add_argument("--serial-steps", type=int, default=3,
                    help="steps of the one-at-a-time comparison (sweep workload)")
    ap.add_argument("--instances", type=int, default=512,
                    help="trap instances of the sweep workload (the first k of the 512-instance sweep)")
    ap.add_argument("--tree-n", type=int, default=1 << 20, help="particles of the tree workload")
    ap.add_argument("--tree-methods", default="",
                    help="comma-separated subset of the tree workload's methods (default: all)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)  # at least three untimed warm-up steps
    if args.impl == "reference":
        if args.workload == "sweep512":
            return run_reference_sweep(args)
        if args.workload == "tree1m":
            return run_reference_tree(args)
        return run_reference(args)
    if args.workload == "sweep512":
        return run_sweep(args)
    if args.workload == "tree1m":
        return run_tree(args)
    return run_amk(args)


if __name__ == "__main__":
    sys.exit(main())
