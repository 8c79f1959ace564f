"""Multi-GPU runs are independent replicas: the only exchange is the final
aggregate (max of the timed intervals, sum of the work). Checked with two
gloo ranks on the host."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        times, counts = bench.reduce_over_ranks([10.0 + rank, 5.0 * (rank + 1)], [100 * (rank + 1), 7])
        q.put((rank, times, counts))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_aggregate_max_time_and_summed_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, times, counts in out:
        assert times == [11.0, 10.0]     # max over ranks of each interval
        assert counts == [300, 14]       # sum over ranks of each count
