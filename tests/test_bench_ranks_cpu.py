"""The bench's replica bookkeeping across ranks (two gloo processes on the
CPU): the job time is the slowest rank's, the work the sum over ranks."""
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


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    st = {"pair_evals": 1000 * (rank + 1), "moves": 10 * (rank + 1), "accepted": 3 + rank, "stages_attempted": 7}
    ms, tot = bench.aggregate_ranks(5.0 + rank, st, dist, "cpu")
    q.put((rank, ms, tot))
    dist.barrier()
    dist.destroy_process_group()


def test_aggregate_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, tot in out:
        assert ms == 6.0
        assert tot == {"pair_evals": 3000, "moves": 30, "accepted": 7, "stages_attempted": 14}


def test_aggregate_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    st = {"pair_evals": 5, "moves": 1}
    assert bench.aggregate_ranks(2.5, st, None, "cpu") == (2.5, st)
