"""Host logic of the multi-rank bench on CPU: two gloo ranks agree on the
slowest rank's step time and on the whole-job rate (replicas: every rank runs
the full workload, no collective on the data path)."""
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


def _rank(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(times[rank], dist, "cpu")
        out[rank] = (t, bench.whole_job_rate(1000, world, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    times = [120.0, 180.0]
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, times, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    t, rate = res[0]
    assert t == pytest.approx(180.0)
    assert rate == pytest.approx(2 * 1000 / 0.180)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(5.0, None, "cpu") == 5.0
    assert bench.whole_job_rate(523776, 1, 1000.0) == pytest.approx(523776.0)
