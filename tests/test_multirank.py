"""Host logic of the multi-process bench on CPU (gloo, world size 2): the
slowest rank's time is what every rank reports; one sweep is partitioned
across the ranks by the per-instance cost model (every instance exactly
once, load within Graham's LPT bound); and the per-instance results gathered
at the end arrive on rank 0 in instance order. The per-instance "results"
come from a CPU stand-in (kinetic energy and particle count of each
instance's initial state), so no GPU is touched."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_INST = 48


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _standin_row(inst):
    pos, vel, sp, p = inst
    m = np.where(sp == 0, 1.67262192369e-27, 9.1093837015e-31)
    return len(pos), float(0.5 * np.sum(m[:, None] * vel ** 2))


def _worker(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from amk import partition
    w, r, _ = bench.dist_setup()
    ms = 10.0 + 5.0 * rank  # rank 1 is the slowest
    slowest = bench.max_over_ranks(ms, w, torch.device("cpu"))
    insts = bench.make_sweep(n_inst=N_INST, seed=2024, method_split=8192)
    mine, imb = bench.sweep_share(insts, w, r)
    rows = [_standin_row(insts[i]) for i in mine]
    gathered = partition.gather_instance_rows(mine, rows, len(insts), w, r)
    parts = [None] * world
    dist.all_gather_object(parts, mine)
    out.put((r, w, slowest, parts, imb, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_partition_one_sweep_and_gather_in_instance_order():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted([q.get(timeout=180) for _ in range(2)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, ROOT)
    import bench
    from amk import partition
    insts = bench.make_sweep(n_inst=N_INST, seed=2024, method_split=8192)
    costs = [partition.instance_cost(len(i[0]), int(i[3].coulomb_method)) for i in insts]
    for r, w, slowest, parts, imb, gathered in results:
        assert w == 2 and slowest == 15.0
        # both ranks hold the same assignment; every instance exactly once
        assert parts == results[0][3]
        flat = sorted(i for part in parts for i in part)
        assert flat == list(range(N_INST))
        # Graham's bound for LPT: max load <= mean load + the largest single cost
        ld = partition.loads(costs, parts)
        assert max(ld) <= sum(ld) / 2 + max(costs) + 1e-6
        assert imb == max(ld) / (sum(ld) / 2)
    # rank 0 holds every instance's row, in instance order
    gathered = results[0][5]
    assert results[1][5] is None
    assert gathered == [_standin_row(i) for i in insts]


def test_lpt_partition_bounds_on_one_process():
    sys.path.insert(0, os.path.join(ROOT, "antimatter-kernel_b200"))
    from amk import partition
    rng = np.random.default_rng(5)
    sizes = (10 ** rng.uniform(2, 5, 512)).astype(int)
    costs = [partition.instance_cost(n, "allpairs" if n < 8192 else "fast-multipole") for n in sizes]
    for world in (1, 2, 3, 4, 8):
        parts = partition.partition_lpt(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(512))
        ld = partition.loads(costs, parts)
        # list scheduling: the last instance placed on the fullest rank
        # started at or below the mean load
        assert max(ld) <= sum(ld) / world + max(costs) + 1e-6 * max(costs)
    try:
        partition.gather_instance_rows([0, 0], ["a", "b"], 2, 1, 0)
    except ValueError:
        pass
    else:
        raise AssertionError("an instance reported twice must be refused")
