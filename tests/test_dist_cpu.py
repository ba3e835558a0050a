"""The multi-GPU bench path on CPU: world_size 2 over gloo.

For N > 1 every rank advances its own copy of the work (replicas; the path
has no data exchange), the job's time is the maximum over ranks, and the
reported value is all ranks' units over that time.  This checks those
helpers and that every rank takes the same collective steps.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    barrier, max_over_ranks = bench.rank_helpers(world, "cpu")
    barrier()
    t = max_over_ranks(1.0 + rank)          # rank 1 is the slower one
    out.put((rank, t, bench.replica_value(1000.0, world, t)))
    barrier()
    dist.destroy_process_group()


def test_replicas_time_is_max_over_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v in res:
        assert t == 2.0                      # every rank sees the slowest rank's time
        assert v == pytest.approx(1000.0 * world / 2.0)


def test_replica_value_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_value(4.0e9, 1, 2.0) == 2.0e9
