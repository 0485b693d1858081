"""The N > 1 path (independent replicas) on CPU: two gloo ranks shard
independent chips, reduce their timings (max) and work (sum) the way
bench.py does, and every chip lands on exactly one rank."""
import os
import socket

import pytest

from hotspot_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    chips = list(range(10))
    mine = replicas.shard(chips, rank, world)
    elapsed = 1.0 + rank          # rank 1 is the slower one
    work = float(sum(mine))
    t, w = replicas.reduce_timing(elapsed, work, dist)
    out[rank] = (mine, t, w)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    import torch.multiprocessing as mp
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    (m0, t0, w0), (m1, t1, w1) = out[0], out[1]
    assert sorted(m0 + m1) == list(range(10)) and not set(m0) & set(m1)
    assert t0 == t1 == 2.0                 # max over ranks
    assert w0 == w1 == float(sum(range(10)))


def test_single_process_passthrough():
    assert replicas.reduce_timing(3.0, 7.0, None) == (3.0, 7.0)
    assert replicas.shard([1, 2, 3], 0, 1) == [1, 2, 3]
