"""Multi-rank path of bench.py on CPU (gloo, world size 2): every rank runs its
own solve (distinct seeds, weak scaling, no collective on the data path); the
job rate is the sum of all ranks' DOF-updates over the maximum of the ranks'
device times."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    seconds = [1.0, 2.5][rank]
    units = [10.0, 30.0][rank]
    rate, tmax, total = bench.aggregate(dist, seconds, units)
    q.put((rank, rate, tmax, total, bench.rank_seed(3, rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_aggregate_is_sum_over_max():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, tmax, total, seed in out:
        assert tmax == 2.5 and total == 40.0
        assert rate == pytest.approx(16.0)
    assert out[0][4] != out[1][4]  # independent solves per rank


def test_single_rank_aggregate():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate(None, 2.0, 8.0) == (4.0, 2.0, 8.0)
