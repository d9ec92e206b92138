"""The N > 1 path of bench.py on the host: two gloo ranks (127.0.0.1) run its barrier and reductions; the whole-job
value is every rank's certified fits over the slowest rank's time, the same on every rank."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    bench.barrier_sync(ws)
    value, tmax = bench.replica_value(50 + rank, 2.0 + rank, ws)
    q.put((rank, value, tmax, bench.sum_over_ranks(1, ws)))
    bench.barrier_sync(ws)
    dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps), [p.exitcode for p in ps]
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, value, tmax, n in out:
        assert tmax == 3.0 and n == 2.0
        assert value == pytest.approx((50 + 51) / 3.0)
