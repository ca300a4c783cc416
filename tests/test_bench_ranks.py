"""The N > 1 path of bench.py on the CPU.  The step does not shard: N GPUs
run N independent replicas, joined only by a barrier and by the slowest
rank's timing (an all-reduce MAX).  That reduction runs here as two gloo
ranks; the reference arm's rule (rank 0 alone runs and prints) is checked
without a process group."""
import argparse
import datetime
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    got = bench.max_over_ranks([1.0 + rank, 5.0 - rank, 3.0], "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    # every rank ends with the slowest rank's figures
    assert results[0] == results[1] == [2.0, 5.0, 3.0]


def test_max_over_ranks_without_a_process_group():
    import bench
    assert bench.max_over_ranks([1.5, 2.5], "cpu") == [1.5, 2.5]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    # returns before any work (no oracle, no workload) on ranks other than 0
    assert bench.run_reference(argparse.Namespace()) == 0
