"""bench.py's multi-GPU mode runs independent replicas (the path has no exchange
step); the only cross-rank steps are a barrier and the max over ranks of the
device times.  Here two gloo ranks on CPU run that reduction and the whole-job
value formula."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
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
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        ms = 100.0 + 25.0 * rank                 # each rank's own device time
        worst = bench.max_over_ranks(ms, dist, "cpu")
        out[rank] = (worst, bench.replica_value(16 * 4096 * 4096, world, 12, worst))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 125.0
    assert res[0][1] == pytest.approx(2 * 16 * 4096 * 4096 * 12 / 0.125)


def test_single_process_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.replica_value(10, 1, 4, 2.0) == pytest.approx(10 * 4 / 2e-3)
