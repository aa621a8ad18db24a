"""bench.py's N>1 path on CPU: two gloo ranks, each a replica, aggregate the
way the benchmark does (bytes summed, time = max over ranks)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # replica r moved (r+1) GB in 10*(r+1) ms and ran 3 steps
        b, ms, extra = bench.aggregate(float(rank + 1) * 1e9, 10.0 * (rank + 1), (3.0,))
        bench.barrier()
        q.put((rank, b, ms, extra))
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, b, ms, extra in res:
        assert b == pytest.approx(3e9)     # bytes summed over replicas
        assert ms == pytest.approx(20.0)   # time = max over ranks
        assert extra == [pytest.approx(6.0)]


def test_aggregation_single_process_is_identity():
    import bench
    assert not (dist.is_available() and dist.is_initialized())
    b, ms, extra = bench.aggregate(5.0, 2.0, (1.0,))
    assert (b, ms, extra) == (5.0, 2.0, [1.0])
    assert torch.tensor(1.0).item() == 1.0
