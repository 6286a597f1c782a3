"""The multi-GPU form of bench.py runs independent replicas ("replicas only":
the operator path has no exchange step).  Its only collective is the
max-over-ranks of the timed region; this runs it on two gloo ranks (CPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = 1.0 + rank  # rank 1 is the slowest
        t_job = bench.job_seconds(t, world)
        out[rank] = (t_job, bench.replica_throughput(100, world, t_job))
    finally:
        dist.destroy_process_group()


def test_job_time_is_max_over_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == pytest.approx(2.0) and res[1][0] == pytest.approx(2.0)
    assert res[0][1] == pytest.approx(100 * 2 / 2.0)
