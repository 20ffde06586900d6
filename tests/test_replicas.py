"""bench.py --gpus N runs independent replicas; the only collectives are the
barrier and the MAX/SUM reductions of the timing. Exercised here with two
gloo ranks on the CPU (127.0.0.1 rendezvous)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    import bench
    ms = [10.0, 25.0][rank]
    cells = [1000, 3000][rank]
    dist.barrier()
    value, max_ms = bench.replica_value(ms, cells, 7, dist, "cpu")
    out[rank] = (value, max_ms)
    dist.destroy_process_group()


def test_two_rank_replica_aggregation():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        value, max_ms = out[r]
        assert max_ms == 25.0
        assert value == pytest.approx((1000 + 3000) * 7 / 25e-3)


def test_single_rank_value():
    sys.path.insert(0, ROOT)
    import bench
    v, ms = bench.replica_value(10.0, 1000, 5)
    assert ms == 10.0 and v == pytest.approx(1000 * 5 / 10e-3)
