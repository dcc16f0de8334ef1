"""bench.py --gpus N runs N independent replicas (the path shards by
instance, no data crosses ranks): the job value is the sum of the ranks'
cell-iterations over the slowest rank's time.  The reduction that forms it,
run by two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, work = bench.combine_ranks(dist, 10.0 + 5 * rank, 1000 * (rank + 1), device="cpu")
        out[rank] = (t, work)
    finally:
        dist.destroy_process_group()


def test_replica_reduction_two_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    # slowest rank's time, total work, the same on every rank
    assert res[0] == res[1] == (15.0, 3000.0)


def test_single_rank_passes_through():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.combine_ranks(None, 12.5, 77) == (12.5, 77)
