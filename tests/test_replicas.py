"""Multi-rank plumbing of bench.py on CPU: two gloo ranks, each an
independent replica (the path does not shard), reduced as the bench reduces
them -- total units over the slowest rank's time."""
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as td
    sys.path.insert(0, REPO)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        value, ms_max, units = bench.replica_throughput(td, 1000 * (rank + 1), 10.0 + rank, device="cpu")
        out.put((rank, value, ms_max, units))
        td.barrier()
    finally:
        td.destroy_process_group()


def test_two_replicas_reduce_to_units_over_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, ms_max, units in got:
        assert ms_max == pytest.approx(11.0)
        assert units == pytest.approx(3000.0)
        assert value == pytest.approx(3000.0 / 11e-3)


def test_single_rank_is_the_identity():
    sys.path.insert(0, REPO)
    import bench
    value, ms_max, units = bench.replica_throughput(None, 500, 2.0)
    assert (value, ms_max, units) == (500 / 2e-3, 2.0, 500)
