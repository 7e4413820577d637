"""The multi-rank path of bench.py (one replica per rank, weak scaling) on
CPU: two gloo ranks on 127.0.0.1 reduce their timings the way the GPU ranks
do -- units summed over ranks, time the max over ranks."""
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


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [120.0, 180.0][rank]
    units = [1.0e9, 3.0e9][rank]
    value, mx = bench.aggregate(units, ms, dist, "cpu")
    out.put((rank, value, mx))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_max_time_and_total_units():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, mx in res:
        assert mx == pytest.approx(180.0)
        assert value == pytest.approx(4.0e9 / 0.180)


def test_single_rank_aggregate_is_local():
    sys.path.insert(0, ROOT)
    import bench
    value, mx = bench.aggregate(2.0e9, 250.0)
    assert mx == 250.0 and value == pytest.approx(8.0e9)
