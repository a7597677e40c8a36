"""Multi-GPU runs are independent frame replicas (one process per GPU, no
collective on the data path): the job's throughput is the units of all ranks
over the slowest rank's time.  Checked with world size 2 on the gloo backend
(CPU) through bench.aggregate, the function bench.py reduces with."""
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


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    # rank r processed 1000 * (r + 1) subsets in 10 * (r + 1) ms
    t, u = bench.aggregate(10.0 * (rank + 1), 1000.0 * (rank + 1), world, "cpu")
    q.put((rank, t, u))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregate_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    # every rank sees the max time and the summed units
    assert res == [(0, 20.0, 3000.0), (1, 20.0, 3000.0)]


def test_replica_aggregate_single():
    import bench
    assert bench.aggregate(12.5, 7.0, 1, "cpu") == (12.5, 7.0)
