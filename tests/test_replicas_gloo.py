"""Host-side logic of the multi-GPU benchmark (replicas only: no data-path
collective) on two gloo ranks on CPU: the max-over-ranks duration and the
whole-job rate."""
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


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    local = [12.5, 20.0][rank]
    t = bench.reduce_max(dist, local, device="cpu")
    rate = bench.aggregate_rate(world, 256 ** 3, 10, t / 1e3)
    out[rank] = (t, rate)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_two_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        t, rate = out[r]
        assert t == 20.0
        assert rate == pytest.approx(2 * 256 ** 3 * 10 / 0.020)
