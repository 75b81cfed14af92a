"""bench.py --gpus N runs N independent replicas (the path does not shard;
no collective on the data path): the only multi-rank steps are the barrier
and the max over ranks of the timed steps.  Checked with two gloo ranks on
the CPU."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    dist.barrier()
    ms = bench.max_over_ranks(times[rank], dist, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ms, bench.job_value(world, 1_000_000, ms / 5)))


def test_two_replicas_take_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    times = [120.0, 150.0]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [150.0, 150.0]
    # 2 replicas x 1e6 samples in 5 steps of 30 ms
    assert all(r[2] == pytest.approx(2 * 1e6 / 0.030 / 1e6) for r in res)
