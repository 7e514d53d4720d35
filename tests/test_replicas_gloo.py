"""bench.py --gpus N runs N independent replicas; the host logic that turns
the ranks' numbers into the job's (slowest rank's time, units summed over
ranks) is exercised here with two gloo ranks on the CPU."""
import os
import socket

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms, units = bench.reduce_over_ranks(dist, 10.0 + 5.0 * rank, 1000 * (rank + 1), "cpu")
    q.put((rank, ms, units))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_reduce_time_and_units():
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
    assert out == [(0, 15.0, 3000.0), (1, 15.0, 3000.0)]


def test_single_process_passthrough():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(None, 12.5, 77, "cpu") == (12.5, 77)
