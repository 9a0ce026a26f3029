"""Host logic of the multi-process bench on CPU (gloo, world size 2): the
slowest rank's time is what every rank reports, and the sweep workload gives
each rank its own instances (no data-path collective)."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    w, r, _ = bench.dist_setup()
    ms = 10.0 + 5.0 * rank  # rank 1 is the slowest
    slowest = bench.max_over_ranks(ms, w, torch.device("cpu"))
    sizes = [len(i[0]) for i in bench.make_sweep(n_inst=6, seed=2024 + r, method_split=None)]
    gathered = [None] * world
    dist.all_gather_object(gathered, sizes)
    out.put((r, w, slowest, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_report_the_slowest_rank_and_shard_the_sweep():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, slowest, gathered in results:
        assert w == 2
        assert slowest == 15.0
        assert gathered[0] != gathered[1]  # each rank's sweep has its own instances
