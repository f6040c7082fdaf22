"""The N > 1 timing rule of bench.py on CPU ranks (gloo, world size 2): every
rank reports its own time, the job's time is the slowest rank's, and the
whole-job value counts the units of all replicas."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
    q.put((rank, ms, bench.weak_value(world, 1000, 5, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_weak_value():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, ms, value in out:
        assert ms == 20.0
        assert value == pytest.approx(2 * 1000 * 5 / 0.020)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5, 1) == 7.5
    assert bench.weak_value(1, 100, 10, 1000.0) == pytest.approx(1000.0)
