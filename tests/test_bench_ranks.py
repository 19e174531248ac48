"""The multi-GPU plumbing of bench.py, on the CPU: with N ranks the set's integrals are dealt
round-robin (each exactly once, no collective on the data path) and only the timings and counts are
reduced after the timed region (max of times, sum of counts).  world_size 2 over gloo."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    names = ['g%02d' % i for i in range(41)]
    mine = bench.assign(names, rank, world)
    mx, sm = bench.reduce_max_sum([10.0 + rank, 1.0], [len(mine), 100.0*(rank + 1)], world)
    q.put((rank, mine, mx, sm))
    dist.destroy_process_group()


def test_two_ranks_deal_every_integral_once_and_reduce():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, m0, mx0, sm0), (_, m1, mx1, sm1) = out
    assert sorted(m0 + m1) == ['g%02d' % i for i in range(41)] and not set(m0) & set(m1)
    assert mx0 == mx1 == [11.0, 1.0]
    assert sm0 == sm1 == [41.0, 300.0]
