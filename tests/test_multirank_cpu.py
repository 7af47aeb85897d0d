"""The multi-GPU path shards the batch per rank with no collective on the data
path (products are independent); the only collectives are the barrier and the
max-over-ranks step time. This CPU test runs that host logic with the gloo
backend at world size 2: each rank draws its own seeded shard, and the
reported time is the maximum over ranks."""
import os
import socket
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    a, b = bench.make_inputs(4, 64, rank)
    local_ms = 1.0 + rank  # rank 1 is the slow one
    worst = bench.reduce_max(local_ms, dist, torch.device("cpu"))
    dist.barrier()
    q.put((rank, float(a.sum()), float(b.sum()), worst))
    dist.destroy_process_group()


def test_two_rank_sharding_and_max_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert out[0][1] != out[1][1]  # each rank has its own shard of the batch
    assert out[0][3] == out[1][3] == 2.0  # whole-job time = slowest rank
