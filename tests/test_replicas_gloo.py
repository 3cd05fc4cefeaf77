"""Multi-GPU runs are independent replicas (the iteration of one block does
not shard); the only cross-rank step is the reduction of the timings, max
over ranks for seconds per step and sum for cell updates.  Checked here with
two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    secs = [0.25, 0.40][rank]
    cells = [1.0e8, 3.0e8][rank]
    q.put((rank, bench.over_ranks(secs, "max", dist, "cpu"), bench.over_ranks(cells, "sum", dist, "cpu")))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timings_reduce_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm in out:
        assert mx == pytest.approx(0.40)
        assert sm == pytest.approx(4.0e8)
